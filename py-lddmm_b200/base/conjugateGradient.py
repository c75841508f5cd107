"""Linear conjugate gradient for `Kernel.solve` (the reference's `Kernel.solve` calls its own linearcg,
base/kernelFunctions.py:676-680; same call signature, `linearcg(op, b, iterMax, x0, param, verb)`).

Hestenes-Stiefel CG for op(x) = b with op symmetric positive definite (a -> K(x) a, whose kernel sums run on the
GPU). It starts from x0 (zero by default) and stops when the residual norm |b - op(x)| falls to `tol` times |b|,
when the curvature p.op(p) is no longer positive, or after iterMax operator applications. Arrays may be numpy
arrays or torch tensors; inner products are read back as Python floats.
"""
import logging

import numpy as np


def _dot(u, v):
    return float((u * v).sum())


def linearcg(op, b, iterMax=100, x0=None, param=None, verb=False, tol=1e-10):
    apply = op if param is None else (lambda v: op(v, param))
    if x0 is None:
        x = b * 0
        r = b * 1
    else:
        x = x0 * 1
        r = b - apply(x)
    bnorm = np.sqrt(_dot(b, b))
    if bnorm == 0.0:
        return x
    p = r * 1
    rr = _dot(r, r)
    for k in range(iterMax):
        if np.sqrt(rr) <= tol * bnorm:
            break
        q = apply(p)
        curv = _dot(p, q)
        if not curv > 0.0:
            logging.info(f'linearcg: non-positive curvature {curv:.3e} at step {k}; returning the current iterate')
            break
        step = rr / curv
        x = x + step * p
        r = r - step * q
        rr_next = _dot(r, r)
        p = r + (rr_next / rr) * p
        rr = rr_next
        if verb:
            logging.info(f'linearcg step {k + 1}: relative residual {np.sqrt(rr) / bnorm:.3e}')
    return x
