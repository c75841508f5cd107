"""Linear conjugate gradient used by `Kernel.solve` (reference: base/conjugateGradient.py:351-409).

Solves op(x) = b for a symmetric positive operator (the kernel sum a -> K(x) a runs on the GPU) with the
reference's stopping rules: |r|^2 < 1e-10 at start, step alpha * mean|p| < 1e-10, or a relative change of the
quadratic energy below 1e-20.
"""
import logging

import numpy as np


def linearcg(op, b, iterMax=100, x0=None, param=None, verb=False):
    apply = (lambda v: op(v)) if param is None else (lambda v: op(v, param))
    x = np.zeros(np.shape(b)) if x0 is None else x0
    z = apply(x) - 2 * b
    ener = (z * x).sum()
    old = ener
    r = -z - b
    mu = None
    p = None
    for i in range(iterMax):
        if i == 0:
            mu = (r * r).sum()
            if mu < 1e-10:
                return x
            p = r
        else:
            mu_old = mu
            mu = (r * r).sum()
            p = r + (mu / mu_old) * p
        q = apply(p)
        alpha = mu / (p * q).sum()
        x = x + alpha * p
        r = r - alpha * q
        z = z + alpha * q
        ener = (z * x).sum()
        if verb and i % 10 == 0:
            logging.info('iter {0:d} ener = {1:.6f} error = {2:.15f}'.format(i + 1, float(ener),
                                                                          float(((apply(x) - b) ** 2).sum())))
        if alpha * np.mean(np.fabs(p)) < 1e-10:
            return x
        if np.fabs(ener - old) < 1e-20 * np.fabs(old):
            return x
        old = ener
    return x
