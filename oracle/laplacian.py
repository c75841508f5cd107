"""Float64 CPU restatement of the Laplacian (Matern) kernel operators (one width sigma, KP = -1).

Reference: base/kernelFunctions_util.py -- the polynomial tables c_, c1_, c2_ and lapPol / lapPolDiff /
lapPolDiff2 (:20-56), the numba functors lap_fun (:92-96), lap_fun_diff (:197-203), lap_fun_diffT (:239-243),
lap_fun_ddiff (:309-314), and the width scalings of applyK_numba (:452-466), applyDiffKT_numba (:774-793),
applyDiffK_numba (:655-680), applyDDiffK_numba (:1092-1129) and applyDiv_numba (:606-620).

With u = |y - x| / sigma and E = exp(-u):
  K       = P0(u) E                                   (P0 = lapPol of the order)
  grad_y  = -P1(u) E (y - x) / sigma^2                (P1 = lapPolDiff)
  Hessian = [P2(u) (y-x)(y-x)^T / sigma^2 - P1(u) I] E / sigma^2   (P2 = lapPolDiff2)
The operators below are the Gaussian ones of oracle/kernels.py with these factors.

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py).
"""
import types

import numpy as np
from numba import njit, prange

# Polynomial coefficients in increasing degree, rows = order 0..4 (base/kernelFunctions_util.py:20-37).
P0 = np.array([[1, 0, 0, 0, 0],
               [1, 1, 0, 0, 0],
               [1, 1, 1 / 3, 0, 0],
               [1, 1, 0.4, 1 / 15, 0],
               [1, 1, 3 / 7, 2 / 21, 1 / 105]], dtype=np.float64)
P1 = np.array([[0, 0, 0, 0, 0],
               [1, 0, 0, 0, 0],
               [1 / 3, 1 / 3, 0, 0, 0],
               [1 / 5, 1 / 5, 1 / 15, 0, 0],
               [1 / 7, 1 / 7, 2 / 35, 1 / 105, 0]], dtype=np.float64)
P2 = np.array([[0, 0, 0, 0, 0],
               [0, 0, 0, 0, 0],
               [1 / 3, 0, 0, 0, 0],
               [1 / 15, 1 / 15, 0, 0, 0],
               [1 / 35, 1 / 35, 1 / 105, 0, 0]], dtype=np.float64)


@njit(cache=True)
def _poly(c, u):
    return c[0] + u * (c[1] + u * (c[2] + u * (c[3] + u * c[4])))


@njit(parallel=True, cache=True)
def _apply_k(y, x, a, inv_s, c0):
    n, m, d = y.shape[0], x.shape[0], a.shape[1]
    out = np.zeros((n, d))
    for k in prange(n):
        acc = np.zeros(d)
        for l in range(m):
            u = np.sqrt((y[k, 0] - x[l, 0]) ** 2 + (y[k, 1] - x[l, 1]) ** 2 + (y[k, 2] - x[l, 2]) ** 2) * inv_s
            e = _poly(c0, u) * np.exp(-u)
            for j in range(d):
                acc[j] += e * a[l, j]
        out[k] = acc
    return out


@njit(parallel=True, cache=True)
def _apply_diff_kt(y, x, p, a, inv_s, c1, mode, w):
    n, m = y.shape[0], x.shape[0]
    out = np.zeros((n, 3))
    for k in prange(n):
        acc = np.zeros(3)
        for l in range(m):
            d0, d1, d2 = y[k, 0] - x[l, 0], y[k, 1] - x[l, 1], y[k, 2] - x[l, 2]
            u = np.sqrt(d0 * d0 + d1 * d1 + d2 * d2) * inv_s
            e = _poly(c1, u) * np.exp(-u)
            c = p[k, 0] * a[l, 0] + p[k, 1] * a[l, 1] + p[k, 2] * a[l, 2]
            if mode >= 1:
                c += a[k, 0] * p[l, 0] + a[k, 1] * p[l, 1] + a[k, 2] * p[l, 2]
            if mode == 2:
                c -= 2.0 * w * (a[k, 0] * a[l, 0] + a[k, 1] * a[l, 1] + a[k, 2] * a[l, 2])
            f = e * c
            acc[0] += f * d0
            acc[1] += f * d1
            acc[2] += f * d2
        out[k] = -inv_s * inv_s * acc
    return out


@njit(parallel=True, cache=True)
def _apply_ddiff(x, nn, a, p, inv_s, c1, c2):
    n = x.shape[0]
    out = np.zeros((n, 3))
    is2 = inv_s * inv_s
    for k in prange(n):
        acc = np.zeros(3)
        for l in range(n):
            d0, d1, d2 = x[k, 0] - x[l, 0], x[k, 1] - x[l, 1], x[k, 2] - x[l, 2]
            q0, q1, q2 = p[k, 0] - p[l, 0], p[k, 1] - p[l, 1], p[k, 2] - p[l, 2]
            u = np.sqrt(d0 * d0 + d1 * d1 + d2 * d2) * inv_s
            ex = np.exp(-u)
            na = nn[k, 0] * a[l, 0] + nn[k, 1] * a[l, 1] + nn[k, 2] * a[l, 2]
            g2 = _poly(c2, u) * ex * na * (d0 * q0 + d1 * q1 + d2 * q2) * is2
            g1 = _poly(c1, u) * ex * na
            acc[0] += g2 * d0 - g1 * q0
            acc[1] += g2 * d1 - g1 * q1
            acc[2] += g2 * d2 - g1 * q2
        out[k] = is2 * acc
    return out


@njit(parallel=True, cache=True)
def _apply_diff_k1and2(x, a1, a2, inv_s, c1):
    n = x.shape[0]
    out = np.zeros((n, 3))
    for k in prange(n):
        acc = np.zeros(3)
        for l in range(n):
            d0, d1, d2 = x[k, 0] - x[l, 0], x[k, 1] - x[l, 1], x[k, 2] - x[l, 2]
            u = np.sqrt(d0 * d0 + d1 * d1 + d2 * d2) * inv_s
            g = _poly(c1, u) * np.exp(-u) * (d0 * (a1[k, 0] - a1[l, 0]) + d1 * (a1[k, 1] - a1[l, 1])
                                               + d2 * (a1[k, 2] - a1[l, 2]))
            acc[0] += g * a2[l, 0]
            acc[1] += g * a2[l, 1]
            acc[2] += g * a2[l, 2]
        out[k] = -inv_s * inv_s * acc
    return out


@njit(parallel=True, cache=True)
def _apply_div(y, x, a, inv_s, c1):
    n, m = y.shape[0], x.shape[0]
    out = np.zeros((n, 1))
    for k in prange(n):
        acc = 0.0
        for l in range(m):
            d0, d1, d2 = y[k, 0] - x[l, 0], y[k, 1] - x[l, 1], y[k, 2] - x[l, 2]
            u = np.sqrt(d0 * d0 + d1 * d1 + d2 * d2) * inv_s
            acc += _poly(c1, u) * np.exp(-u) * (d0 * a[l, 0] + d1 * a[l, 1] + d2 * a[l, 2])
        out[k, 0] = -inv_s * inv_s * acc
    return out


def _f(v):
    return np.ascontiguousarray(v, dtype=np.float64)


def apply_k(y, x, a, sigma, order=3):
    """z_k = sum_l P0(u) e^-u a_l (lap_fun, base/kernelFunctions_util.py:92-96)."""
    a2 = _f(a)
    if a2.ndim == 1:
        a2 = a2[:, None]
    return _apply_k(_f(y), _f(x), a2, 1.0 / sigma, P0[order])


def apply_diff_kt(y, x, p, a, sigma, sym=False, lddmm=False, regweight=1.0, order=3):
    """z_k = sum_l -(y_k - x_l)/sigma^2 P1(u) e^-u c_kl (lap_fun_diffT, base/kernelFunctions_util.py:239-243)."""
    mode = 2 if lddmm else (1 if sym else 0)
    return _apply_diff_kt(_f(y), _f(x), _f(p), _f(a), 1.0 / sigma, P1[order], mode, float(regweight))


def apply_ddiff_k11and12(x, n, a, p, sigma, order=3):
    """sum_l (n_k.a_l) [P2 (D.Dp) D / sigma^4 - P1 Dp / sigma^2] e^-u (lap_fun_ddiff, :309-314)."""
    return _apply_ddiff(_f(x), _f(n), _f(a), _f(p), 1.0 / sigma, P1[order], P2[order])


def apply_diff_k1and2(x, a1, a2, sigma, order=3):
    """sum_l -(D.(a1_k - a1_l))/sigma^2 P1 e^-u a2_l (lap_fun_diff, :197-203; option '1and2' :672-675)."""
    return _apply_diff_k1and2(_f(x), _f(a1), _f(a2), 1.0 / sigma, P1[order])


def apply_divergence(y, x, a, sigma, order=3):
    """sum_l -((y_k - x_l).a_l)/sigma^2 P1 e^-u (applyDiv_numba with lap_fun_diff, :606-620)."""
    return _apply_div(_f(y), _f(x), _f(a), 1.0 / sigma, P1[order])


def ops(order):
    """The operator set of one order, with the signatures of oracle/kernels.py (for oracle/shooting.py)."""
    return types.SimpleNamespace(
        apply_k=lambda y, x, a, s: apply_k(y, x, a, s, order),
        apply_diff_kt=lambda y, x, p, a, s, **kw: apply_diff_kt(y, x, p, a, s, order=order, **kw),
        apply_ddiff_k11and12=lambda x, n, a, p, s: apply_ddiff_k11and12(x, n, a, p, s, order),
        apply_diff_k1and2=lambda x, a1, a2, s: apply_diff_k1and2(x, a1, a2, s, order),
        apply_divergence=lambda y, x, a, s: apply_divergence(y, x, a, s, order))
