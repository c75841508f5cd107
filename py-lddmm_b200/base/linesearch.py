"""Line searches of the optimiser protocol (reference: base/linesearch.py:4-282).

Same arguments, return tuple (t, fc, gc, phi(t), phi(0), gradient at t) and acceptance tests as the reference;
the objective and gradient evaluations are the caller's (`opt.updateTry`, `opt.getGradient(update=...)`),
which run on the GPU. Scalars compared here are FP64 values read back from the device.
"""
import logging

from scipy.optimize._linesearch import scalar_search_wolfe2


def _slope(opt, g, pk, euclidean):
    dp = opt.dotProduct_euclidean if euclidean else opt.dotProduct
    return -dp(g, [pk])[0]


def line_search_weak_wolfe(opt, pk, gfk=None, old_fval=None, old_old_fval=None, c1=0.001, c2=0.9, amax=None,
                           maxiter=100, euclidean=True, t_init=1.):
    """Bisection / quadratic-interpolation search for the weak Wolfe conditions (base/linesearch.py:66-163):
    Armijo  phi(t) < phi(0) + c1 t phi'(0) g,  curvature  phi'(t) > c2 phi'(0) g  (g = opt.gradCoeff)."""
    counts = {'f': 0, 'g': 0}
    last_grad = [None]

    def phi(t):
        counts['f'] += 1
        return opt.updateTry(pk, t)

    def dphi(t):
        counts['g'] += 1
        last_grad[0] = opt.getGradient(opt.gradCoeff, update=[pk, t])
        return _slope(opt, last_grad[0], pk, euclidean)

    if gfk is None:
        gfk = opt.getGradient(opt.gradCoeff)
    d0 = _slope(opt, gfk, pk, euclidean)
    if old_fval is None:
        old_fval = phi(0)
    g = getattr(opt, 'gradCoeff', 1)
    lo, hi = 0.0, 0.0
    t = t_init
    n_f_max = 100
    it = 0
    n_grad = 0
    f = phi(t)
    while it < n_f_max and n_grad < maxiter:
        armijo = f < old_fval + c1 * t * d0 * g
        if armijo:
            df = dphi(t)
            n_grad += 1
            if df > c2 * d0 * g:
                break
            lo = t
        else:
            hi = t
        if hi < 1e-16:
            t *= 2
        elif armijo:
            t = 0.5 * (lo + hi)
        else:
            tq = -(t ** 2 * d0) / (2 * (f - old_fval - t * d0))
            t = max(0.9 * lo + 0.1 * hi, min(0.5 * (lo + hi), tq))
        f = phi(t)
        it += 1

    if n_grad == maxiter:
        logging.warning(f'weak-Wolfe search: {maxiter} gradients spent without meeting the curvature test; '
                        'halving the step until the decrease test holds')
        last_grad[0] = None
        while it < n_f_max:
            if f < old_fval + c1 * t * d0 * g:
                dphi(t)
                break
            t /= 2
            f = phi(t)
            it += 1

    if it == n_f_max:
        logging.warning(f'weak-Wolfe search gave up after {n_f_max} trial steps (objective {f:.6g} against {old_fval:.6g})')
        t = None
    return t, counts['f'], counts['g'], f, old_fval, last_grad[0]


def line_search_goldstein_price(opt, pk, gfk=None, old_fval=None, old_old_fval=None, c1=0.001, c2=0.9, amax=None,
                                maxiter=100, euclidean=True, t_init=1.):
    """Goldstein-Price bracketing on the mean slope (base/linesearch.py:4-63)."""
    counts = {'f': 0}

    def phi(t):
        counts['f'] += 1
        return opt.updateTry(pk, t)

    if gfk is None:
        gfk = opt.getGradient(opt.gradCoeff)
    d0 = _slope(opt, gfk, pk, euclidean)
    if old_fval is None:
        old_fval = phi(0)
    lo, hi = 0.0, 0.0
    t = 1.
    f = phi(t)
    r = (f - old_fval) / t
    it = 0
    while it < maxiter:
        if r < c1 * d0:
            if r > c2 * d0:
                break
            lo = t
        else:
            hi = t
        t = t * 2 if hi < 1e-10 else 0.5 * (lo + hi)
        f = phi(t)
        r = (f - old_fval) / t
        it += 1
    if it == maxiter:
        logging.warning(f'Goldstein-Price search gave up after {maxiter} trial steps')
        t = None
    return t, counts['f'], 0, f, old_fval, None


def line_search_wolfe(opt, pk, gfk=None, old_fval=None, old_old_fval=None, c1=0.001, c2=0.9, amax=None,
                      maxiter=100, euclidean=True, t_init=1.):
    """Strong Wolfe search through scipy's scalar_search_wolfe2 (base/linesearch.py:164-282)."""
    counts = {'f': 0, 'g': 0}
    last_grad = [None]

    def phi(t):
        counts['f'] += 1
        return opt.updateTry(pk, t)

    def dphi(t):
        counts['g'] += 1
        last_grad[0] = opt.getGradient(opt.gradCoeff, update=[pk, t])
        return _slope(opt, last_grad[0], pk, euclidean)

    if gfk is None:
        gfk = opt.getGradient(opt.gradCoeff)
    d0 = _slope(opt, gfk, pk, euclidean)
    t, f, old_fval, _ = scalar_search_wolfe2(phi, dphi, old_fval, old_old_fval, d0, c1, c2, amax, None,
                                             maxiter=maxiter)
    return t, counts['f'], counts['g'], f, old_fval, last_grad[0]
