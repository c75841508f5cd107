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


class RowGather:
    """All-gather of every rank's (rows, width) block into the full (n, width) array, with the padded send buffer and
    the receive buffer allocated once and reused by every step (a rank's block has at most `chunk` rows; the padding
    rows of the last ranks land past row n and are dropped)."""

    def __init__(self, n, width=3, dtype=torch.float64, device=None, group=None):
        self.n, self.group = n, group
        world = dist.get_world_size(group)
        self.chunk = row_chunk(n, world)
        self.send = torch.zeros((self.chunk, width), dtype=dtype, device=device)
        self.recv = torch.empty((world * self.chunk, width), dtype=dtype, device=device)

    def __call__(self, local, out=None):
        self.send[:local.shape[0]].copy_(local)
        dist.all_gather_into_tensor(self.recv, self.send, group=self.group)
        if out is None:
            return self.recv[:self.n].clone()
        out.copy_(self.recv[:self.n])
        return out


def all_gather_rows(local, n, group=None):
    """Concatenate every rank's (rows, 3) block (rows <= chunk, zero-padded for the collective) into (n, 3)."""
    return RowGather(n, local.shape[1], local.dtype, local.device, group)(local)


def all_reduce_fp64(value, group=None):
    """Sum of a float64 scalar (device tensor) over the ranks of `group` (energies)."""
    v = value.to(torch.float64).reshape(1).clone()
    dist.all_reduce(v, op=dist.ReduceOp.SUM, group=group)
    return v[0]


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


def library_k_rows(K, origin):
    """Rows r0..r1 of K(x) a on the GPU (lddmm_apply_k with the row range as targets)."""
    sigma = float(np.asarray(K.sigma).ravel()[0])
    o = nat.origin_arg(origin)

    def k_rows(x, a, r0, r1):
        n, nr = x.shape[0], r1 - r0
        out = torch.empty((nr, 3), dtype=torch.float64, device=x.device)
        if nr == 0:
            return out
        y = x[r0:r1].contiguous()
        ws, wsb = nat.workspace(nr, n, K.precision)
        nat.check(nat.lib().lddmm_apply_k(nat.ptr(y), nr, nat.ptr(x), nat.ptr(a), n, sigma, K.code, o, nat.ptr(out),
                                          K.precision, ws, wsb, nat.stream_ptr()), 'apply_k')
        return out
    return k_rows


def sharded_second_order_shoot(X0, A0, timeStep, step_rows, group=None, gather=None):
    """Geodesic shooting with the rows of every step sharded over the ranks of `group`; returns the full (xt, at)
    (T+1, n, 3) on every rank (secondOrderEvolution, base/pointEvolution.py:385-472)."""
    world, rank = dist.get_world_size(group), dist.get_rank(group)
    T = int(np.round(1.0 / timeStep))
    n = X0.shape[0]
    r0, r1 = row_range(n, world, rank)
    gather = gather or RowGather(n, 3, X0.dtype, X0.device, group)
    xt = torch.empty((T + 1, n, 3), dtype=X0.dtype, device=X0.device)
    at = torch.empty_like(xt)
    xt[0], at[0] = X0, A0
    for t in range(T):
        x1, a1 = step_rows(xt[t], at[t], r0, r1, timeStep)
        gather(x1, xt[t + 1])
        gather(a1, at[t + 1])
    return xt, at


def sharded_second_order_adjoint(xt, at, px1, pa1, timeStep, adjoint_rows, group=None, gather=None):
    """Adjoint sweep (secondOrderCovector, base/pointEvolution.py:489-552) with the rows of every step sharded;
    returns the full (pxt, pat) on every rank."""
    world, rank = dist.get_world_size(group), dist.get_rank(group)
    T = xt.shape[0] - 1
    n = xt.shape[1]
    r0, r1 = row_range(n, world, rank)
    gather = gather or RowGather(n, 3, xt.dtype, xt.device, group)
    pxt = torch.empty_like(xt)
    pat = torch.empty_like(xt)
    pxt[T], pat[T] = px1, pa1
    for t in range(T - 1, -1, -1):
        p0, q0 = adjoint_rows(xt[t], at[t], pxt[t + 1], pat[t + 1], r0, r1, timeStep)
        gather(p0, pxt[t])
        gather(q0, pat[t])
    return pxt, pat


def sharded_kinetic(X0, A0, k_rows, group=None, gather=None):
    """(0.5 a0.K(x0)a0 as an FP64 device scalar summed over the ranks, full K(x0)a0 on every rank): the kinetic term
    of the second-order objective (base/secondOrderPointSetMatching.py:113-148) with its rows sharded."""
    world, rank = dist.get_world_size(group), dist.get_rank(group)
    n = X0.shape[0]
    r0, r1 = row_range(n, world, rank)
    ka = k_rows(X0, A0, r0, r1)
    e = all_reduce_fp64(0.5 * (A0[r0:r1] * ka).sum(), group)
    gather = gather or RowGather(n, 3, X0.dtype, X0.device, group)
    return e, gather(ka)


def sharded_second_order_gradient(X0, A0, px1, timeStep, step_rows, adjoint_rows, k_rows, group=None):
    """The second-order objective's deformation part and gradient with every sum sharded by rows: shooting, the FP64
    kinetic energy, the adjoint sweep from the end-point covector px1 (pa1 = 0) and da0 = K(x0)a0 - pa_0
    (base/secondOrderPointSetMatching.py:379-483). Returns (kinetic energy, xt, at, da0), identical on every rank."""
    gather = RowGather(X0.shape[0], 3, X0.dtype, X0.device, group)
    xt, at = sharded_second_order_shoot(X0, A0, timeStep, step_rows, group, gather)
    e, ka0 = sharded_kinetic(X0, A0, k_rows, group, gather)
    _, pat = sharded_second_order_adjoint(xt, at, px1, torch.zeros_like(px1), timeStep, adjoint_rows, group, gather)
    return e, xt, at, ka0 - pat[0]
