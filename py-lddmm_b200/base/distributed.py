"""Row-sharded geodesic shooting and adjoint over torch.distributed (one process per GPU).

Every all-pairs sum of a time step is independent per target row, so rank r computes the rows
[r*chunk, min(n, (r+1)*chunk)) of the new state from the full, replicated state of the previous step, and one
all-gather (NCCL over NVLink on GPUs) assembles the next full state on every rank: 2 x 3 x 8 x n bytes per step
(forward: x, a; adjoint: px, pa), microseconds next to the O(n^2) sums. Results are bitwise identical on every rank
and equal to the single-GPU trajectory up to the summation order of the shards (the same kernels run on each row
range). The step functions are pluggable so that the host-side logic (row ranges, padding, gathers, time loop)
runs on CPU `gloo` ranks in the tests; on GPUs they are the library's row-range step entry points.
"""
import numpy as np
import torch
import torch.distributed as dist

from . import _native as nat


def row_chunk(n, world):
    return (n + world - 1) // world


def row_range(n, world, rank):
    c = row_chunk(n, world)
    r0 = min(n, rank * c)
    return r0, min(n, r0 + c)


def all_gather_rows(local, n, group=None):
    """Concatenate every rank's (rows, 3) block (rows <= chunk, zero-padded for the collective) into (n, 3)."""
    world = dist.get_world_size(group)
    c = row_chunk(n, world)
    buf = torch.zeros((c, local.shape[1]), dtype=local.dtype, device=local.device)
    buf[:local.shape[0]] = local
    out = torch.empty((world * c, local.shape[1]), dtype=local.dtype, device=local.device)
    dist.all_gather_into_tensor(out, buf, group=group)
    return out[:n].contiguous()


def library_step_rows(K, origin):
    """Row-range second-order step on the GPU (lddmm_second_order_step_rows)."""
    sigma = float(np.asarray(K.sigma).ravel()[0])
    o = nat.origin_arg(origin)

    def step(x, a, r0, r1, dt):
        n, nr = x.shape[0], r1 - r0
        x1 = torch.empty((nr, 3), dtype=torch.float64, device=x.device)
        a1 = torch.empty_like(x1)
        ws, wsb = nat.workspace(max(nr, 1), n, K.precision)
        nat.check(nat.lib().lddmm_second_order_step_rows(nat.ptr(x), nat.ptr(a), n, r0, nr, sigma, K.code, float(dt),
                                                         o, nat.ptr(x1), nat.ptr(a1), K.precision, ws, wsb,
                                                         nat.stream_ptr()), 'second_order_step_rows')
        return x1, a1
    return step


def library_adjoint_rows(K, origin):
    """Row-range second-order adjoint step on the GPU (lddmm_second_order_adjoint_step_rows)."""
    sigma = float(np.asarray(K.sigma).ravel()[0])
    o = nat.origin_arg(origin)

    def step(x, a, px, pa, r0, r1, dt):
        n, nr = x.shape[0], r1 - r0
        p0 = torch.empty((nr, 3), dtype=torch.float64, device=x.device)
        q0 = torch.empty_like(p0)
        ws, wsb = nat.workspace(max(nr, 1), n, K.precision)
        nat.check(nat.lib().lddmm_second_order_adjoint_step_rows(nat.ptr(x), nat.ptr(a), nat.ptr(px), nat.ptr(pa), n,
                                                                 r0, nr, sigma, K.code, float(dt), o, nat.ptr(p0),
                                                                 nat.ptr(q0), K.precision, ws, wsb, nat.stream_ptr()),
                  'second_order_adjoint_step_rows')
        return p0, q0
    return step


def sharded_second_order_shoot(X0, A0, timeStep, step_rows, group=None):
    """Geodesic shooting with the rows of every step sharded over the ranks of `group`; returns the full (xt, at)
    (T+1, n, 3) on every rank (secondOrderEvolution, base/pointEvolution.py:385-472)."""
    world, rank = dist.get_world_size(group), dist.get_rank(group)
    T = int(np.round(1.0 / timeStep))
    n = X0.shape[0]
    r0, r1 = row_range(n, world, rank)
    xt = torch.empty((T + 1, n, 3), dtype=X0.dtype, device=X0.device)
    at = torch.empty_like(xt)
    xt[0], at[0] = X0, A0
    for t in range(T):
        x1, a1 = step_rows(xt[t], at[t], r0, r1, timeStep)
        xt[t + 1] = all_gather_rows(x1, n, group)
        at[t + 1] = all_gather_rows(a1, n, group)
    return xt, at


def sharded_second_order_adjoint(xt, at, px1, pa1, timeStep, adjoint_rows, group=None):
    """Adjoint sweep (secondOrderCovector, base/pointEvolution.py:489-552) with the rows of every step sharded;
    returns the full (pxt, pat) on every rank."""
    world, rank = dist.get_world_size(group), dist.get_rank(group)
    T = xt.shape[0] - 1
    n = xt.shape[1]
    r0, r1 = row_range(n, world, rank)
    pxt = torch.empty_like(xt)
    pat = torch.empty_like(xt)
    pxt[T], pat[T] = px1, pa1
    for t in range(T - 1, -1, -1):
        p0, q0 = adjoint_rows(xt[t], at[t], pxt[t + 1], pat[t + 1], r0, r1, timeStep)
        pxt[t] = all_gather_rows(p0, n, group)
        pat[t] = all_gather_rows(q0, n, group)
    return pxt, pat
