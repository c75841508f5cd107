"""Limited-memory BFGS driver of the optimiser protocol (reference: base/bfgs.py:55-313).

The optimisable object `opt` provides getVariable, objectiveFun, updateTry, acceptVarTry, getGradient and
optionally dotProduct(_euclidean), addProd, prod, copyDir, startOfIteration, endOfIteration, endOfProcedure,
gradEps, gradCoeff, epsMax, burnIn -- the same protocol as the reference. The two-loop recursion, the initial
step 1/|q| at the first iteration, the stopping rules (|obj - obj_old| < 1e-7 after burn-in, |grad| < gradEps)
and the reset-on-failed-line-search logic follow the reference; directions live wherever `opt` keeps them
(device tensors for the B200 matching classes).
"""
import logging
import time
from copy import deepcopy

import numpy as np
import torch

from .linesearch import line_search_wolfe, line_search_weak_wolfe, line_search_goldstein_price


def _dot(x, ys):
    return [float((x * y).sum()) for y in ys]


def bfgs(opt, verb=True, maxIter=1000, TestGradient=False, epsInit=0.01, memory=25, Wolfe=True,
         lineSearch='Weak_Wolfe'):
    for need in ('getVariable', 'objectiveFun', 'updateTry', 'acceptVarTry', 'getGradient'):
        if not hasattr(opt, need):
            logging.error('bfgs: the object lacks part of the optimiser protocol (%s)', need)
            return
    line_search = {'Wolfe': line_search_wolfe, 'Goldstein_Price': line_search_goldstein_price,
                   'Weak_Wolfe': line_search_weak_wolfe}.get(lineSearch, line_search_weak_wolfe)
    dot = getattr(opt, 'dotProduct_euclidean', None) or getattr(opt, 'dotProduct', None) or _dot
    # optional: (u, v) -> u.v as a device scalar, used by the two-loop recursion (no host synchronisation)
    dot_dev = getattr(opt, 'dotProduct_device', None)
    # optional: (gradient, history) -> the two-loop recursion's direction in one call, or None to run it here
    fused_direction = getattr(opt, 'lbfgs_direction', None)
    # optional: (objective, |gradient|^2) -> the first step along the gradient, or None for 1 / |gradient|
    initial_step = getattr(opt, 'initial_step', None)
    addProd = getattr(opt, 'addProd', lambda x, y, a: x + a * y)
    prod = getattr(opt, 'prod', lambda x, a: a * x)
    copyDir = getattr(opt, 'copyDir', deepcopy)
    stopCondition = getattr(opt, 'stopCondition', lambda: True)
    if hasattr(opt, 'startOptim'):
        opt.startOptim()
    if hasattr(opt, 'gradEps'):
        gradEps = opt.gradEps
    elif hasattr(opt, 'options') and 'gradEps' in opt.options:
        gradEps = opt.options['gradEps']
    else:
        gradEps = None
    gradCoeff = getattr(opt, 'gradCoeff', 1.0)
    epsMax = getattr(opt, 'epsMax', 1.)
    burnIn = getattr(opt, 'burnIn', 0)
    eps = epsInit
    opt.converged = False
    if getattr(opt, 'reset', False):
        opt.obj = None
    obj = opt.objectiveFun()
    opt.reset = False
    logging.info(f'bfgs start: objective {obj:.6g}')

    history = []
    it = 0
    diffVar = None
    grdOld = None
    obj_old = None
    gval = None

    def finish():
        if hasattr(opt, 'endOfProcedure'):
            opt.endOfProcedure()
        elif hasattr(opt, 'endOfIteration'):
            opt.endOfIteration()

    t_iter = time.process_time()
    while it < maxIter:
        t0 = time.process_time()
        if hasattr(opt, 'startOfIteration'):
            opt.startOfIteration()
        if opt.reset:
            opt.obj = None
            obj = opt.objectiveFun()
            if verb:
                logging.info(f'bfgs restart: objective re-evaluated as {obj:.6g}')
            obj_old = None
            gval = None
        grd = opt.getGradient(gradCoeff) if gval is None else gval

        if TestGradient:
            dirfoo = opt.randomDir() if hasattr(opt, 'randomDir') else np.random.normal(size=np.shape(grd))
            epsfoo = 1e-8
            o1 = opt.updateTry(dirfoo, epsfoo, obj - 1e8)
            o2 = opt.updateTry(dirfoo, -epsfoo, obj - 1e8)
            [gd] = dot(grd, [dirfoo])
            logging.info(f'gradient check along a random direction: finite difference {(o1 - o2) / (2 * epsfoo):.4f}, '
                         f'analytic {-gd * gradCoeff:.4f}')

        q = None
        if not opt.reset and it > 0:
            history.append([diffVar, addProd(grd, grdOld, -1)])
            if len(history) > memory:
                history.pop(0)
            if fused_direction is not None:
                q = fused_direction(grd, history)
            if q is None:
                q = copyDir(grd)
                # the two-loop recursion; with `dot_dev` (device scalars) it runs without reading anything back
                d = dot_dev or (lambda u, v: dot(u, [v])[0])
                rho, alpha = [], []
                for s_k, y_k in reversed(history):
                    rho.append(1 / d(y_k, s_k))
                    alpha.append(rho[-1] * d(s_k, q))
                    q = addProd(q, y_k, -alpha[-1])
                rho.reverse()
                alpha.reverse()
                s_k, y_k = history[-1]
                c = d(s_k, y_k) / d(y_k, y_k)
                if dot_dev is not None:
                    c = torch.where(c < 1e-10, torch.ones_like(c), c)
                elif c < 1e-10:
                    c = 1
                q = prod(q, c)
                for k, (s_k, y_k) in enumerate(history):
                    beta = rho[k] * d(y_k, q)
                    q = addProd(q, s_k, alpha[k] - beta)
        else:
            history = []
            q = copyDir(grd)

        grd2 = dot(grd, [grd])[0]
        grdTry = np.sqrt(np.maximum(1e-20, dot(q, [q])[0]))
        dir0 = copyDir(q)
        t_init = 1. / grdTry if (it == 0 or opt.reset) else 1.
        if it == 0 and not opt.reset and initial_step is not None:
            t_hint = initial_step(obj, grd2)
            if t_hint is not None:
                t_init = t_hint
        grdOld = copyDir(grd)

        if it == 0 or it == burnIn:
            if gradEps is None:
                gradEps = max(0.001 * np.sqrt(grd2), 0.0001)
            else:
                gradEps = min(gradEps, 0.0001 * np.sqrt(grd2))
            logging.info(f'bfgs: stop when the gradient norm falls below {gradEps:.6g}')

        if it < burnIn:
            Wolfe = False
            eps = epsInit
        elif Wolfe:
            eps = 1.
        else:
            eps = min(eps, epsMax / grdTry)

        eps, fc, gc, phi_star, old_fval, gval = line_search(opt, dir0, gfk=grd, old_fval=obj, old_old_fval=obj_old,
                                                            c1=1e-4, c2=0.9, amax=None, t_init=t_init, maxiter=10)
        if eps is not None:
            diffVar = prod(dir0, -eps)
            obj_old = obj
            opt.acceptVarTry()
            obj = phi_star
            newreset = False
        else:
            logging.info('bfgs: the line search found no acceptable step')
            if opt.reset:
                logging.info('bfgs: second failed line search in a row after a restart; stopping')
                opt.converged = False
                finish()
                break
            newreset = True
            gval = None

        if obj_old is not None and np.fabs(obj - obj_old) < 1e-7 and stopCondition():
            logging.info(f'bfgs step {it + 1:d}: objective {obj:.6g}, step {eps:.4g}, |gradient| {np.sqrt(grd2):.4g}')
            if it > burnIn or opt.reset:
                logging.info('bfgs: objective change below 1e-7; converged')
                opt.converged = True
                finish()
                break
            newreset = True

        now = time.process_time()
        if verb or it == maxIter:
            e_s = 'None' if eps is None else f'{eps:.5f}'
            logging.info(f'bfgs step {it + 1:d}: objective {obj:.6g}, step {e_s}, |gradient| {np.sqrt(grd2):.4g}, '
                         f'{now - t0:.3f} s')
        t_iter = now

        if np.sqrt(grd2) < gradEps and stopCondition():
            logging.info('bfgs: gradient norm below the threshold; converged')
            opt.converged = True
            finish()
            break
        eps = np.minimum(100 * eps, epsMax) if eps is not None else epsMax
        opt.reset = newreset
        if hasattr(opt, 'endOfIteration'):
            opt.endOfIteration()
        if not opt.reset:
            it += 1

    if it == maxIter and hasattr(opt, 'endOfProcedure'):
        opt.endOfProcedure()
    if hasattr(opt, 'endOptim'):
        opt.endOptim()
    return opt.getVariable()
