"""Float64 CPU restatement of landmark shooting and its adjoint (no affine part, no splines).

Reference: base/pointEvolution.py. Every function takes `ops`, the kernel operator set: the Gaussian one of
oracle/kernels.py by default, or oracle.laplacian.ops(order). TEST INFRASTRUCTURE ONLY (see oracle/__init__.py).
"""
import types

import numpy as np
from numba import njit, prange

from . import kernels as _gauss

GAUSS = types.SimpleNamespace(apply_k=_gauss.apply_k, apply_diff_kt=_gauss.apply_diff_kt,
                              apply_ddiff_k11and12=_gauss.apply_ddiff_k11and12,
                              apply_diff_k1and2=_gauss.apply_diff_k1and2,
                              apply_divergence=_gauss.apply_divergence)


def landmark_direct_evolution_euler(x0, at, sigma, ops=GAUSS):
    """x_{t+1} = x_t + dt K(x_t) a_t, dt = 1/T  (base/pointEvolution.py:88-164)."""
    T = at.shape[0]
    dt = 1.0 / T
    xt = np.zeros((T + 1,) + x0.shape)
    xt[0] = x0
    for t in range(T):
        xt[t + 1] = xt[t] + dt * ops.apply_k(xt[t], xt[t], at[t], sigma)
    return xt


def landmark_hamiltonian_gradient(x0, at, px1, sigma, regweight, ops=GAUSS):
    """Backward sweep p_t = p_{t+1} + dt DK^T_lddmm(x_t; p_{t+1}, a_t); dat_t = 2 w a_t - p_{t+1}
    (base/pointEvolution.py:167-236). Returns (dat, xt, pxt)."""
    T = at.shape[0]
    dt = 1.0 / T
    xt = landmark_direct_evolution_euler(x0, at, sigma, ops)
    pxt = np.zeros((T + 1,) + x0.shape)
    pxt[T] = px1
    for t in range(T - 1, -1, -1):
        px = pxt[t + 1]
        pxt[t] = px + dt * ops.apply_diff_kt(xt[t], xt[t], px, at[t], sigma, lddmm=True, regweight=regweight)
    dat = 2.0 * regweight * at - pxt[1:]
    return dat, xt, pxt


def second_order_evolution(x0, a0, sigma, timeStep, ops=GAUSS):
    """x += dt K(x) a, a -= dt DK^T(x; a, a), T = round(1/timeStep) steps of size timeStep
    (base/pointEvolution.py:385-472). Returns (xt, at)."""
    T = int(np.round(1.0 / timeStep))
    xt = np.zeros((T + 1,) + x0.shape)
    at = np.zeros((T + 1,) + x0.shape)
    xt[0], at[0] = x0, a0
    for k in range(T):
        x, a = xt[k], at[k]
        zx = ops.apply_k(x, x, a, sigma)
        za = -ops.apply_diff_kt(x, x, a, a, sigma)
        xt[k + 1] = x + timeStep * zx
        at[k + 1] = a + timeStep * za
    return xt, at


def landmark_epdiff(T, x0, a0, sigma, point_set=None, normals=None, jacobian=False, ops=GAUSS):
    """landmarkEPDiff (base/pointEvolution.py:320-382): T steps of 1/T of x += dt K(x) a, a -= dt DK^T(x; a, a)
    (momentum kept for steps 0..T-1), with a point set carried by y += dt K(x, y) a, normals by
    n -= dt DK^T(x; n, a) and the log-Jacobian by J += dt div(K a)(x). Returns the reference's list
    [xt, at, (yt), (nt), (Jt)], or (xt, at) with nothing extra requested."""
    T = int(T)
    dt = 1.0 / T
    xt = np.zeros((T + 1,) + x0.shape)
    at = np.zeros((T,) + x0.shape)
    xt[0], at[0] = x0, a0
    out_y = out_n = out_j = None
    if point_set is not None:
        out_y = np.zeros((T + 1,) + point_set.shape)
        out_y[0] = point_set
    if normals is not None:
        out_n = np.zeros((T + 1,) + normals.shape)
        out_n[0] = normals
    if jacobian:
        out_j = np.zeros((T + 1, x0.shape[0], 1))
    for k in range(T):
        x, a = xt[k], at[k]
        xt[k + 1] = x + dt * ops.apply_k(x, x, a, sigma)
        if k < T - 1:
            at[k + 1] = a - dt * ops.apply_diff_kt(x, x, a, a, sigma)
        if out_y is not None:
            out_y[k + 1] = out_y[k] + dt * ops.apply_k(out_y[k], x, a, sigma)
        if out_n is not None:
            out_n[k + 1] = out_n[k] - dt * ops.apply_diff_kt(x, x, out_n[k], a, sigma)
        if out_j is not None:
            out_j[k + 1] = out_j[k] + dt * ops.apply_divergence(x, x, a, sigma).reshape(-1, 1)
    extra = [v for v in (out_y, out_n, out_j) if v is not None]
    return (xt, at) if not extra else [xt, at] + extra


def second_order_gradient(x0, a0, px1, pa1, sigma, timeStep, ops=GAUSS):
    """Adjoint of second-order shooting (base/pointEvolution.py:489-618):
    px <- px + dt [DK^T_sym(x; px, a) - DDK11and12(x; a, a, pa)], pa <- pa + dt [K(x) px - DK1and2(x; pa, a)],
    da0 = K(x0) a0 - pa_0. Returns dict(da0, xt, at, pxt, pat)."""
    T = int(np.round(1.0 / timeStep))
    xt, at = second_order_evolution(x0, a0, sigma, timeStep, ops)
    pxt = np.zeros((T + 1,) + x0.shape)
    pat = np.zeros((T + 1,) + x0.shape)
    pxt[T], pat[T] = px1, pa1
    for t in range(T - 1, -1, -1):
        px, pa, x, a = pxt[t + 1], pat[t + 1], xt[t], at[t]
        zpx = ops.apply_diff_kt(x, x, px, a, sigma, sym=True) - ops.apply_ddiff_k11and12(x, a, a, pa, sigma)
        zpa = ops.apply_k(x, x, px, sigma) - ops.apply_diff_k1and2(x, pa, a, sigma)
        pxt[t] = px + timeStep * zpx
        pat[t] = pa + timeStep * zpa
    da0 = ops.apply_k(x0, x0, a0, sigma) - pat[0]
    return dict(da0=da0, xt=xt, at=at, pxt=pxt, pat=pat)


@njit(parallel=True, cache=True)
def _so_step_rows(x, a, rows, inv_s2):
    r = rows.shape[0]
    zx = np.zeros((r, 3))
    za = np.zeros((r, 3))
    inv2s2 = 0.5 * inv_s2
    for i in prange(r):
        k = rows[i]
        for l in range(x.shape[0]):
            d0, d1, d2 = x[k, 0] - x[l, 0], x[k, 1] - x[l, 1], x[k, 2] - x[l, 2]
            e = np.exp(-(d0 * d0 + d1 * d1 + d2 * d2) * inv2s2)
            c = e * (a[k, 0] * a[l, 0] + a[k, 1] * a[l, 1] + a[k, 2] * a[l, 2])
            zx[i, 0] += e * a[l, 0]
            zx[i, 1] += e * a[l, 1]
            zx[i, 2] += e * a[l, 2]
            za[i, 0] += c * d0
            za[i, 1] += c * d1
            za[i, 2] += c * d2
    return zx, za * inv_s2


def second_order_step_rows(x, a, rows, sigma):
    """One secondOrderEvolution step restricted to the target rows `rows`, against every point
    (base/pointEvolution.py:433-449): returns (K(x)a, -DK^T(x; a, a)) at those rows, so that x1 = x + dt zx and
    a1 = a + dt za. -DK^T(x; a, a)_k = sum_l (x_k - x_l)/sigma^2 e_kl (a_k.a_l)."""
    return _so_step_rows(np.ascontiguousarray(x, np.float64), np.ascontiguousarray(a, np.float64),
                         np.ascontiguousarray(rows, np.int64), 1.0 / sigma ** 2)


@njit(parallel=True, cache=True)
def _so_adjoint_rows(x, a, px, pa, rows, inv_s2):
    r = rows.shape[0]
    zpx = np.zeros((r, 3))
    zpa = np.zeros((r, 3))
    inv2s2 = 0.5 * inv_s2
    for i in prange(r):
        k = rows[i]
        for l in range(x.shape[0]):
            d0, d1, d2 = x[k, 0] - x[l, 0], x[k, 1] - x[l, 1], x[k, 2] - x[l, 2]
            q0, q1, q2 = pa[k, 0] - pa[l, 0], pa[k, 1] - pa[l, 1], pa[k, 2] - pa[l, 2]
            e = np.exp(-(d0 * d0 + d1 * d1 + d2 * d2) * inv2s2)
            # DK^T_sym(x; px, a): -(x_k - x_l)/sigma^2 e (px_k.a_l + a_k.px_l)
            c1 = (px[k, 0] * a[l, 0] + px[k, 1] * a[l, 1] + px[k, 2] * a[l, 2]
                  + a[k, 0] * px[l, 0] + a[k, 1] * px[l, 1] + a[k, 2] * px[l, 2])
            # DDK11and12(x; a, a, pa): (a_k.a_l) e [(D.Dpa) D / sigma^4 - Dpa / sigma^2]
            c2 = e * (a[k, 0] * a[l, 0] + a[k, 1] * a[l, 1] + a[k, 2] * a[l, 2])
            dq = (d0 * q0 + d1 * q1 + d2 * q2) * inv_s2
            zpx[i, 0] += -e * c1 * d0 * inv_s2 - c2 * (dq * d0 - q0) * inv_s2
            zpx[i, 1] += -e * c1 * d1 * inv_s2 - c2 * (dq * d1 - q1) * inv_s2
            zpx[i, 2] += -e * c1 * d2 * inv_s2 - c2 * (dq * d2 - q2) * inv_s2
            # K(x) px - DK1and2(x; pa, a): e px_l + (D.Dpa)/sigma^2 e a_l
            zpa[i, 0] += e * px[l, 0] + dq * e * a[l, 0]
            zpa[i, 1] += e * px[l, 1] + dq * e * a[l, 1]
            zpa[i, 2] += e * px[l, 2] + dq * e * a[l, 2]
    return zpx, zpa


def second_order_adjoint_step_rows(x, a, px, pa, rows, sigma):
    """One secondOrderCovector step restricted to the target rows `rows` (base/pointEvolution.py:539-546):
    zpx = DK^T_sym(x; px, a) - DDK11and12(x; a, a, pa), zpa = K(x) px - DK1and2(x; pa, a) at those rows, so that
    px_prev = px + dt zpx and pa_prev = pa + dt zpa."""
    f = lambda v: np.ascontiguousarray(v, np.float64)   # noqa: E731
    return _so_adjoint_rows(f(x), f(a), f(px), f(pa), np.ascontiguousarray(rows, np.int64), 1.0 / sigma ** 2)
