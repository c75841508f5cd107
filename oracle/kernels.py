"""Float64 CPU restatement of the Gaussian kernel operators (one width sigma, KP = -1).

Reference: base/kernelFunctions_util.py (numba backends) behind base/kernelFunctions.py `Kernel`.
With a single width and the default `ms_exponent = -1` the scale weights s**KP / sum(s**KP) reduce to
1 for K, 1/sigma**2 for first derivatives and 1/sigma**2 (plus the 1/sigma**2 inside the functor) for the
second derivative; the formulas below are written directly in those terms.

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py).
"""
import numpy as np
from numba import njit, prange


@njit(parallel=True, cache=True)
def _apply_k(y, x, a, inv2s2):
    n, m, d = y.shape[0], x.shape[0], a.shape[1]
    out = np.zeros((n, d))
    for k in prange(n):
        acc = np.zeros(d)
        for l in range(m):
            r2 = (y[k, 0] - x[l, 0]) ** 2 + (y[k, 1] - x[l, 1]) ** 2 + (y[k, 2] - x[l, 2]) ** 2
            e = np.exp(-r2 * inv2s2)
            for j in range(d):
                acc[j] += e * a[l, j]
        out[k] = acc
    return out


def apply_k(y, x, a, sigma):
    """z_k = sum_l exp(-|y_k - x_l|^2 / (2 sigma^2)) a_l  (base/kernelFunctions_util.py:451-466)."""
    a2 = np.ascontiguousarray(a, dtype=np.float64)
    if a2.ndim == 1:
        a2 = a2[:, None]
    return _apply_k(np.ascontiguousarray(y, np.float64), np.ascontiguousarray(x, np.float64), a2,
                    0.5 / sigma ** 2)


@njit(parallel=True, cache=True)
def _apply_diff_kt(y, x, p, a, inv2s2, mode, w):
    n, m = y.shape[0], x.shape[0]
    out = np.zeros((n, 3))
    for k in prange(n):
        acc = np.zeros(3)
        for l in range(m):
            d0, d1, d2 = y[k, 0] - x[l, 0], y[k, 1] - x[l, 1], y[k, 2] - x[l, 2]
            e = np.exp(-(d0 * d0 + d1 * d1 + d2 * d2) * inv2s2)
            c = p[k, 0] * a[l, 0] + p[k, 1] * a[l, 1] + p[k, 2] * a[l, 2]
            if mode >= 1:
                c += a[k, 0] * p[l, 0] + a[k, 1] * p[l, 1] + a[k, 2] * p[l, 2]
            if mode == 2:
                c -= 2.0 * w * (a[k, 0] * a[l, 0] + a[k, 1] * a[l, 1] + a[k, 2] * a[l, 2])
            f = e * c
            acc[0] += f * d0
            acc[1] += f * d1
            acc[2] += f * d2
        out[k] = -2.0 * inv2s2 * acc
    return out


def apply_diff_kt(y, x, p, a, sigma, sym=False, lddmm=False, regweight=1.0):
    """z_k = sum_l -(y_k - x_l)/sigma^2 e_kl c_kl with c_kl = p_k.a_l (+ a_k.p_l if sym or lddmm)
    (- 2 regweight a_k.a_l if lddmm)  (base/kernelFunctions_util.py:773-793, gauss_fun_diffT :233)."""
    mode = 2 if lddmm else (1 if sym else 0)
    return _apply_diff_kt(np.ascontiguousarray(y, np.float64), np.ascontiguousarray(x, np.float64),
                          np.ascontiguousarray(p, np.float64), np.ascontiguousarray(a, np.float64),
                          0.5 / sigma ** 2, mode, float(regweight))


@njit(parallel=True, cache=True)
def _apply_ddiff(x, nn, a, p, inv_s2):
    n = x.shape[0]
    out = np.zeros((n, 3))
    inv2s2 = 0.5 * inv_s2
    for k in prange(n):
        acc = np.zeros(3)
        for l in range(n):
            d0, d1, d2 = x[k, 0] - x[l, 0], x[k, 1] - x[l, 1], x[k, 2] - x[l, 2]
            q0, q1, q2 = p[k, 0] - p[l, 0], p[k, 1] - p[l, 1], p[k, 2] - p[l, 2]
            e = np.exp(-(d0 * d0 + d1 * d1 + d2 * d2) * inv2s2)
            c = (nn[k, 0] * a[l, 0] + nn[k, 1] * a[l, 1] + nn[k, 2] * a[l, 2]) * e
            dq = (d0 * q0 + d1 * q1 + d2 * q2) * inv_s2
            acc[0] += c * (dq * d0 - q0)
            acc[1] += c * (dq * d1 - q1)
            acc[2] += c * (dq * d2 - q2)
        out[k] = acc * inv_s2
    return out


def apply_ddiff_k11and12(x, n, a, p, sigma):
    """z_k = sum_l (n_k.a_l) e_kl [ (D.Dp) D / sigma^4 - Dp / sigma^2 ], D = x_k - x_l, Dp = p_k - p_l
    (base/kernelFunctions_util.py:1091-1129 option '11and12', gauss_fun_ddiff :299)."""
    return _apply_ddiff(np.ascontiguousarray(x, np.float64), np.ascontiguousarray(n, np.float64),
                        np.ascontiguousarray(a, np.float64), np.ascontiguousarray(p, np.float64), 1.0 / sigma ** 2)


@njit(parallel=True, cache=True)
def _apply_diff_k1and2(x, a1, a2, inv_s2):
    n = x.shape[0]
    out = np.zeros((n, 3))
    inv2s2 = 0.5 * inv_s2
    for k in prange(n):
        acc = np.zeros(3)
        for l in range(n):
            d0, d1, d2 = x[k, 0] - x[l, 0], x[k, 1] - x[l, 1], x[k, 2] - x[l, 2]
            e = np.exp(-(d0 * d0 + d1 * d1 + d2 * d2) * inv2s2)
            g = d0 * (a1[k, 0] - a1[l, 0]) + d1 * (a1[k, 1] - a1[l, 1]) + d2 * (a1[k, 2] - a1[l, 2])
            f = -e * g
            acc[0] += f * a2[l, 0]
            acc[1] += f * a2[l, 1]
            acc[2] += f * a2[l, 2]
        out[k] = acc * inv_s2
    return out


def apply_diff_k1and2(x, a1, a2, sigma):
    """z_k = sum_l -(D.(a1_k - a1_l))/sigma^2 e_kl a2_l  (base/kernelFunctions_util.py:672-675, gauss_fun_diff :195)."""
    return _apply_diff_k1and2(np.ascontiguousarray(x, np.float64), np.ascontiguousarray(a1, np.float64),
                              np.ascontiguousarray(a2, np.float64), 1.0 / sigma ** 2)


@njit(parallel=True, cache=True)
def _apply_div(y, x, a, inv_s2):
    n, m = y.shape[0], x.shape[0]
    out = np.zeros((n, 1))
    inv2s2 = 0.5 * inv_s2
    for k in prange(n):
        acc = 0.0
        for l in range(m):
            d0, d1, d2 = y[k, 0] - x[l, 0], y[k, 1] - x[l, 1], y[k, 2] - x[l, 2]
            e = np.exp(-(d0 * d0 + d1 * d1 + d2 * d2) * inv2s2)
            acc -= e * (d0 * a[l, 0] + d1 * a[l, 1] + d2 * a[l, 2])
        out[k, 0] = acc * inv_s2
    return out


def apply_divergence(y, x, a, sigma):
    """z_k = sum_l -((y_k - x_l).a_l)/sigma^2 e_kl, shape (N,1)  (base/kernelFunctions_util.py:611-626)."""
    return _apply_div(np.ascontiguousarray(y, np.float64), np.ascontiguousarray(x, np.float64),
                      np.ascontiguousarray(a, np.float64), 1.0 / sigma ** 2)


@njit(parallel=True, cache=True)
def _apply_k_tensor(y, x, ay, ax, by, bx, inv2s2):
    n, m = y.shape[0], x.shape[0]
    out = np.zeros(n)
    for k in prange(n):
        acc = 0.0
        for l in range(m):
            r2 = (y[k, 0] - x[l, 0]) ** 2 + (y[k, 1] - x[l, 1]) ** 2 + (y[k, 2] - x[l, 2]) ** 2
            e = np.exp(-r2 * inv2s2)
            g = by[k, 0] * bx[l, 0] + by[k, 1] * bx[l, 1] + by[k, 2] * bx[l, 2]
            acc += e * (ay[k] * ax[l] + g * g)
        out[k] = acc
    return out


def apply_k_tensor(y, x, ay, ax, betay, betax, sigma):
    """f_k = sum_l e_kl (ay_k ax_l + (betay_k.betax_l)^2)  (base/kernelFunctions_util.py:1475-1506)."""
    c = lambda v: np.ascontiguousarray(v, np.float64)
    return _apply_k_tensor(c(y), c(x), c(ay).ravel(), c(ax).ravel(), c(betay), c(betax), 0.5 / sigma ** 2)


@njit(parallel=True, cache=True)
def _apply_k_mat(y, x, u, inv2s2):
    n, m, d = y.shape[0], x.shape[0], u.shape[2]
    out = np.zeros((n, d))
    for k in prange(n):
        for l in range(m):
            r2 = (y[k, 0] - x[l, 0]) ** 2 + (y[k, 1] - x[l, 1]) ** 2 + (y[k, 2] - x[l, 2]) ** 2
            e = np.exp(-r2 * inv2s2)
            for j in range(d):
                out[k, j] += e * u[k, l, j]
    return out


def apply_k_mat(y, x, u, sigma):
    """f_k = sum_l e_kl u[k, l, :]  (applyK(matrixWeights=True), base/kernelFunctions_util.py:1509-1540)."""
    return _apply_k_mat(np.ascontiguousarray(y, np.float64), np.ascontiguousarray(x, np.float64),
                        np.ascontiguousarray(u, np.float64), 0.5 / sigma ** 2)


@njit(parallel=True, cache=True)
def _apply_diff_k_mat(y, x, beta, inv_s2):
    n, m = y.shape[0], x.shape[0]
    out = np.zeros((n, 3))
    inv2s2 = 0.5 * inv_s2
    for k in prange(n):
        for l in range(m):
            d0, d1, d2 = y[k, 0] - x[l, 0], y[k, 1] - x[l, 1], y[k, 2] - x[l, 2]
            f = -np.exp(-(d0 * d0 + d1 * d1 + d2 * d2) * inv2s2) * beta[k, l] * inv_s2
            out[k, 0] += f * d0
            out[k, 1] += f * d1
            out[k, 2] += f * d2
    return out


def apply_diff_k_mat(y, x, beta, sigma):
    """f_k = sum_l -(y_k - x_l)/sigma^2 e_kl beta[k, l]  (base/kernelFunctions_util.py:1638-1669)."""
    return _apply_diff_k_mat(np.ascontiguousarray(y, np.float64), np.ascontiguousarray(x, np.float64),
                             np.ascontiguousarray(beta, np.float64), 1.0 / sigma ** 2)
