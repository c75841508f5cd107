"""Row-sharded shooting, adjoint and second-order gradient (base/distributed.py) on world-size-2 `gloo` ranks on the
CPU, with the oracle's float64 sums as the per-rank steps: the gathered trajectories, the gradient da0 and the
all-reduced kinetic energy equal the single-process oracle's."""
import os
import sys

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from conftest import PKG, REPO

SIGMA, DT = 0.5, 0.1


def _oracle_steps():
    import oracle as O

    def step(x, a, r0, r1, dt):
        X, A = x.numpy(), a.numpy()
        y = X[r0:r1]
        zx = O.apply_k(y, X, A, SIGMA)
        za = -O.apply_diff_kt(y, X, A[r0:r1], A, SIGMA)
        return torch.from_numpy(y + dt * zx), torch.from_numpy(A[r0:r1] + dt * za)

    def adjoint(x, a, px, pa, r0, r1, dt):
        X, A, PX, PA = x.numpy(), a.numpy(), px.numpy(), pa.numpy()
        zpx = O.apply_diff_kt(X, X, PX, A, SIGMA, sym=True) - O.apply_ddiff_k11and12(X, A, A, PA, SIGMA)
        zpa = O.apply_k(X, X, PX, SIGMA) - O.apply_diff_k1and2(X, PA, A, SIGMA)
        return torch.from_numpy(PX[r0:r1] + dt * zpx[r0:r1]), torch.from_numpy(PA[r0:r1] + dt * zpa[r0:r1])
    return step, adjoint


def _oracle_k_rows(x, a, r0, r1):
    import oracle as O
    X, A = x.numpy(), a.numpy()
    return torch.from_numpy(O.apply_k(X[r0:r1], X, A, SIGMA))


def _worker(rank, world, port, x0, a0, px1, result_path):
    for p in (REPO, PKG):
        if p not in sys.path:
            sys.path.insert(0, p)
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    import torch.distributed as dist
    from base import distributed as dd
    dist.init_process_group('gloo', rank=rank, world_size=world)
    try:
        step, adjoint = _oracle_steps()
        X0, A0 = torch.from_numpy(x0), torch.from_numpy(a0)
        xt, at = dd.sharded_second_order_shoot(X0, A0, DT, step)
        pxt, pat = dd.sharded_second_order_adjoint(xt, at, torch.from_numpy(px1), torch.zeros_like(X0), DT, adjoint)
        e, _, _, da0 = dd.sharded_second_order_gradient(X0, A0, torch.from_numpy(px1), DT, step, adjoint,
                                                        _oracle_k_rows)
        if rank == 0:
            np.savez(result_path, xt=xt.numpy(), at=at.numpy(), pxt=pxt.numpy(), pat=pat.numpy(), da0=da0.numpy(),
                     kinetic=float(e))
        # every rank holds the same gathered trajectory
        h = torch.tensor([float(xt.sum()), float(pxt.sum())], dtype=torch.float64)
        hs = [torch.zeros_like(h) for _ in range(world)]
        dist.all_gather(hs, h)
        assert all(torch.equal(v, hs[0]) for v in hs)
    finally:
        dist.destroy_process_group()


def test_row_ranges_cover_every_row_once():
    from base.distributed import row_range
    for n in (1, 7, 162, 1000):
        for world in (1, 2, 3, 8):
            rows = np.concatenate([np.arange(*row_range(n, world, r)) for r in range(world)])
            assert np.array_equal(rows, np.arange(n))


def test_sharded_shooting_gloo_world2(tmp_path):
    import oracle as O
    from base.syntheticShapes import icosphere, smooth_momenta
    x0, _ = icosphere(2)
    rng = np.random.default_rng(4)
    a0 = smooth_momenta(x0, rng, O.apply_k, sigma_smooth=0.4, sigma_def=SIGMA, vmax=0.3)
    px1 = rng.normal(size=x0.shape)
    out = str(tmp_path / 'res.npz')
    port = 29500 + (os.getpid() % 1000)
    mp.start_processes(_worker, args=(2, port, x0, a0, px1, out), nprocs=2, join=True, start_method='spawn')
    r = np.load(out)
    ref = O.second_order_gradient(x0, a0, px1, np.zeros_like(x0), SIGMA, DT)
    for k in ('xt', 'at', 'pxt', 'pat', 'da0'):
        assert np.allclose(r[k], ref[k], rtol=1e-12, atol=1e-12), k
    assert np.isclose(float(r['kinetic']), 0.5 * (a0 * O.apply_k(x0, x0, a0, SIGMA)).sum(), rtol=1e-13)
