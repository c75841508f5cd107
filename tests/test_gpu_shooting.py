"""Parity of the fused shooting / adjoint kernels with the reference (base/pointEvolution.py).

Tolerance (relative L2 error against float64): FP32 compensated path 2e-5, FP64 path 1e-11.
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN, rel_err

pytestmark = pytest.mark.gpu
TOL = {'float32': 2e-5, 'float64': 1e-11}


def kernel(sigma, dtype):
    from base.kernelFunctions import Kernel
    K = Kernel(name='gauss', sigma=sigma)
    K.pk_dtype = dtype
    return K


@pytest.mark.parametrize('dtype', ['float32', 'float64'])
def test_first_order_vs_reference(dtype):
    from base import pointEvolution as evol
    d = np.load(os.path.join(GOLDEN, 'first_order_L2.npz'))
    K = kernel(float(d['sigma']), dtype)
    st = evol.landmarkDirectEvolutionEuler(d['x0'], d['at'], K)
    assert rel_err(st['xt'], d['xt']) < TOL[dtype]
    dat, xt, pxt = evol.landmarkHamiltonianGradient(d['x0'], d['at'], d['px1'], K, float(d['regweight']),
                                                    getCovector=True)
    assert rel_err(dat, d['dat']) < TOL[dtype]
    assert rel_err(pxt, d['pxt']) < TOL[dtype]


@pytest.mark.parametrize('dtype', ['float32', 'float64'])
def test_second_order_vs_reference(dtype):
    from base import pointEvolution as evol
    d = np.load(os.path.join(GOLDEN, 'second_order_L2.npz'))
    K = kernel(float(d['sigma']), dtype)
    g = evol.secondOrderGradient(d['x0'], d['a0'], d['px1'], d['pa1'], K, float(d['timeStep']))
    for k in ('xt', 'at', 'da0', 'pxt', 'pat'):
        assert rel_err(g[k], d[k]) < TOL[dtype], (k, rel_err(g[k], d[k]))
    fw = evol.secondOrderEvolution(d['x0'], d['a0'], K, float(d['timeStep']))
    assert rel_err(fw['xt'], d['xt']) < TOL[dtype]


@pytest.mark.parametrize('dtype', ['float32', 'float64'])
def test_landmark_epdiff_vs_reference(dtype):
    """landmarkEPDiff with a point set and normals against the reference's output; the Jacobian (which the
    reference's line cannot return: it broadcasts an (N,1) divergence into an (N,) slice) against the oracle."""
    import oracle as O
    from base import pointEvolution as evol
    d = np.load(os.path.join(GOLDEN, 'epdiff_L2.npz'))
    K = kernel(float(d['sigma']), dtype)
    T = int(d['T'])
    xt, at, yt, nt = evol.landmarkEPDiff(T, d['x0'], d['a0'], K, withNormals=d['n0'], withPointSet=d['y0'])
    for k, v in (('xt', xt), ('at', at), ('yt', yt), ('nt', nt)):
        assert v.shape == d[k].shape, k
        assert rel_err(v, d[k]) < TOL[dtype], (k, rel_err(v, d[k]))
    xs, as_ = evol.landmarkEPDiff(T, d['x0'], d['a0'], K)
    assert rel_err(xs, d['xt']) < TOL[dtype] and rel_err(as_, d['at']) < TOL[dtype]
    _, _, Jt = evol.landmarkEPDiff(T, d['x0'], d['a0'], K, withJacobian=True)
    _, _, Jref = O.landmark_epdiff(T, d['x0'], d['a0'], float(d['sigma']), jacobian=True)
    assert Jt.shape == Jref.shape and rel_err(Jt, Jref) < TOL[dtype]


def test_second_order_l4_vs_oracle():
    import oracle as O
    from base import pointEvolution as evol
    from base.syntheticShapes import icosphere, smooth_momenta
    x0, _ = icosphere(4)
    rng = np.random.default_rng(5)
    a0 = smooth_momenta(x0, rng, O.apply_k, sigma_smooth=0.4, sigma_def=0.5, vmax=0.3)
    px1 = rng.normal(0, 0.5, x0.shape)
    pa1 = np.zeros_like(x0)
    ref = O.second_order_gradient(x0, a0, px1, pa1, 0.5, 0.1)
    g = evol.secondOrderGradient(x0, a0, px1, pa1, kernel(0.5, 'float32'), 0.1)
    for k in ('xt', 'at', 'da0', 'pxt', 'pat'):
        assert rel_err(g[k], ref[k]) < 2e-5, (k, rel_err(g[k], ref[k]))


def test_step_entry_points_match_trajectory():
    """The per-step C-ABI calls reproduce the whole-trajectory calls exactly (same kernels, same order)."""
    import torch
    from base import _native as nat
    from base import pointEvolution as evol
    from base.syntheticShapes import icosphere
    x0, _ = icosphere(3)
    rng = np.random.default_rng(6)
    X0 = torch.from_numpy(x0).cuda()
    A0 = torch.from_numpy(rng.normal(0, 0.2, x0.shape)).cuda()
    K = kernel(0.5, 'float32')
    o = nat.centroid(X0)
    xt, at = evol.shoot_second_order(X0, A0, K, 0.1, origin=o)
    x, a = X0.clone(), A0.clone()
    ws, wsb = nat.workspace(x0.shape[0], x0.shape[0])
    for t in range(10):
        x1, a1 = torch.empty_like(x), torch.empty_like(a)
        nat.check(nat.lib().lddmm_second_order_step(nat.ptr(x), nat.ptr(a), x.shape[0], 0.5, 0, 0.1, nat.origin_arg(o),
                                                    nat.ptr(x1), nat.ptr(a1), 0, ws, wsb, nat.stream_ptr()))
        x, a = x1, a1
    assert torch.equal(x, xt[-1]) and torch.equal(a, at[-1])
    px = torch.from_numpy(rng.normal(size=x0.shape)).cuda()
    pa = torch.zeros_like(px)
    pxt, pat, _ = evol.second_order_adjoint(xt, at, px, pa, K, 0.1, origin=o)
    for t in range(9, -1, -1):
        p0, q0 = torch.empty_like(px), torch.empty_like(pa)
        nat.check(nat.lib().lddmm_second_order_adjoint_step(nat.ptr(xt[t]), nat.ptr(at[t]), nat.ptr(px), nat.ptr(pa),
                                                            x.shape[0], 0.5, 0, 0.1, nat.origin_arg(o), nat.ptr(p0),
                                                            nat.ptr(q0), 0, ws, wsb, nat.stream_ptr()))
        px, pa = p0, q0
    assert torch.equal(px, pxt[0]) and torch.equal(pa, pat[0])


def test_first_order_energy_and_euclidean_gradient():
    import torch
    import oracle as O
    from base import pointEvolution as evol
    d = np.load(os.path.join(GOLDEN, 'first_order_L2.npz'))
    K = kernel(0.5, 'float64')
    X0, AT = torch.from_numpy(d['x0']).cuda(), torch.from_numpy(d['at']).cuda()
    e = torch.zeros(1, dtype=torch.float64, device='cuda')
    xt = evol.shoot_first_order(X0, AT, K, regweight=0.8, energy=e)
    T = AT.shape[0]
    ref = sum(0.8 / T * (d['at'][t] * O.apply_k(d['xt'][t], d['xt'][t], d['at'][t], 0.5)).sum() for t in range(T))
    assert abs(float(e) - ref) < 1e-12 * abs(ref)
    pxt, dat = evol.first_order_gradient(xt, AT, torch.from_numpy(d['px1']).cuda(), K, 0.8, euclidean=True)
    for t in range(T):
        g = 2 * 0.8 * d['at'][t] - d['pxt'][t + 1]
        assert rel_err(dat[t].cpu().numpy(), O.apply_k(d['xt'][t], d['xt'][t], g, 0.5)) < 1e-11


def test_first_order_symmetric_kernels_level4():
    """First-order shooting and adjoint at level 4 (2,562 points: several row blocks, so the FP32 symmetric kernels
    credit pairs to both points), FP32 against the oracle: the trajectory, the kinetic energy, the covectors and the
    euclidean gradient (relative L2 2e-5, the FP32 shooting tolerance)."""
    import torch
    import oracle as O
    from base import pointEvolution as evol
    from base.syntheticShapes import icosphere
    x0, _ = icosphere(4)
    rng = np.random.default_rng(21)
    T, w = 5, 0.8
    at = np.stack([O.apply_k(x0, x0, rng.normal(0, 0.02, x0.shape), 0.3) for _ in range(T)])
    px1 = rng.normal(size=x0.shape)
    K = kernel(0.5, 'float32')
    e = torch.zeros(1, dtype=torch.float64, device='cuda')
    AT = torch.from_numpy(at).cuda()
    xt = evol.shoot_first_order(torch.from_numpy(x0).cuda(), AT, K, regweight=w, energy=e)
    dat_ref, xt_ref, pxt_ref = O.landmark_hamiltonian_gradient(x0, at, px1, 0.5, w)
    assert rel_err(xt.cpu().numpy() - x0, xt_ref - x0) < 2e-5
    e_ref = sum(w / T * (at[t] * O.apply_k(xt_ref[t], xt_ref[t], at[t], 0.5)).sum() for t in range(T))
    assert abs(float(e) - e_ref) < 2e-5 * abs(e_ref)
    pxt, dat = evol.first_order_gradient(xt, AT, torch.from_numpy(px1).cuda(), K, w)
    assert rel_err(pxt.cpu().numpy() - px1, pxt_ref - px1) < 2e-5
    assert rel_err(dat.cpu().numpy(), dat_ref) < 2e-5
    _, dat_e = evol.first_order_gradient(xt, AT, torch.from_numpy(px1).cuda(), K, w, euclidean=True)
    for t in range(T):
        g = 2 * w * at[t] - pxt_ref[t + 1]
        assert rel_err(dat_e[t].cpu().numpy(), O.apply_k(xt_ref[t], xt_ref[t], g, 0.5)) < 2e-5


@pytest.mark.parametrize('dtype', ['float32', 'float64'])
def test_row_range_steps_match_whole_steps(dtype):
    """lddmm_second_order_step_rows / _adjoint_step_rows on a row range equal the same rows of the whole step."""
    import torch
    from base import distributed as dd
    from base import _native as nat
    from base import pointEvolution as evol
    from base.syntheticShapes import icosphere
    x0, _ = icosphere(4)
    rng = np.random.default_rng(8)
    X = torch.from_numpy(x0).cuda()
    A = torch.from_numpy(rng.normal(0, 0.01, x0.shape)).cuda()
    PX = torch.from_numpy(rng.normal(size=x0.shape)).cuda()
    PA = torch.from_numpy(rng.normal(0, 0.1, x0.shape)).cuda()
    K = kernel(0.5, dtype)
    o = nat.centroid(X)
    xt, at = evol.shoot_second_order(X, A, K, 0.5, origin=o)            # two steps of size 0.5
    step = dd.library_step_rows(K, o)
    adj = dd.library_adjoint_rows(K, o)
    tol = 1e-6 if dtype == 'float32' else 1e-13
    for r0, r1 in ((0, x0.shape[0]), (100, 1300), (2000, 2562)):
        x1, a1 = step(X, A, r0, r1, 0.5)
        assert rel_err(x1.cpu().numpy(), xt[1, r0:r1].cpu().numpy()) < tol
        assert rel_err(a1.cpu().numpy(), at[1, r0:r1].cpu().numpy()) < tol
    pxt, pat, _ = evol.second_order_adjoint(xt, at, PX, PA, K, 0.5, origin=o, with_da0=False)
    for r0, r1 in ((0, x0.shape[0]), (7, 901)):
        p0, q0 = adj(xt[1], at[1], PX, PA, r0, r1, 0.5)
        assert rel_err(p0.cpu().numpy(), pxt[1, r0:r1].cpu().numpy()) < tol
        assert rel_err(q0.cpu().numpy(), pat[1, r0:r1].cpu().numpy()) < tol


def test_sharded_shooting_nccl_single_rank():
    """The NCCL code path of the sharded driver on one GPU (world size 1) reproduces the unsharded trajectory."""
    import os
    import torch
    import torch.distributed as dist
    from base import distributed as dd
    from base import pointEvolution as evol
    from base import _native as nat
    from base.syntheticShapes import icosphere
    x0, _ = icosphere(3)
    X = torch.from_numpy(x0).cuda()
    A = torch.from_numpy(np.random.default_rng(9).normal(0, 0.01, x0.shape)).cuda()
    K = kernel(0.5, 'float32')
    o = nat.centroid(X)
    os.environ.setdefault('MASTER_ADDR', '127.0.0.1')
    os.environ.setdefault('MASTER_PORT', str(29400 + os.getpid() % 500))
    dist.init_process_group('nccl', rank=0, world_size=1)
    try:
        xt, at = dd.sharded_second_order_shoot(X, A, 0.1, dd.library_step_rows(K, o))
        torch.cuda.synchronize()
    finally:
        dist.destroy_process_group()
    rx, ra = evol.shoot_second_order(X, A, K, 0.1, origin=o)
    assert torch.equal(xt, rx) and torch.equal(at, ra)


@pytest.mark.parametrize('n', [1, 2, 33, 129, 511, 512, 513, 1025, 2049, 5000])
def test_symmetric_adjoint_step_ragged_sizes(n):
    """The whole-step FP32 Gaussian adjoint step evaluates each unordered pair once (pairs_kernel_sym). It must agree
    with the ordered-pair kernel (the same step computed as two row ranges) and with the FP64 oracle at sizes that
    leave partial blocks and tiles, a single block, and blocks whose column partials come from many rows."""
    import torch
    import oracle as O
    from base import distributed as dd
    from base import _native as nat
    rng = np.random.default_rng(n)
    x = rng.uniform(-1, 1, (n, 3))
    a = rng.normal(0, 0.1, (n, 3))
    px = rng.normal(size=(n, 3))
    pa = rng.normal(0, 0.1, (n, 3))
    X, A, PX, PA = (torch.from_numpy(v).cuda() for v in (x, a, px, pa))
    K = kernel(0.5, 'float32')
    o = nat.centroid(X)
    adj = dd.library_adjoint_rows(K, o)
    dt = 0.05
    p_sym, q_sym = adj(X, A, PX, PA, 0, n, dt)
    h = n // 2
    parts = [adj(X, A, PX, PA, r0, r1, dt) for r0, r1 in ((0, h), (h, n)) if r1 > r0]
    p_ord = torch.cat([p for p, _ in parts])
    q_ord = torch.cat([q for _, q in parts])
    zpx, zpa = O.second_order_adjoint_step_rows(x, a, px, pa, np.arange(n), 0.5)
    for got, ref_o, base in ((p_sym, p_ord, px), (q_sym, q_ord, pa)):
        inc, inc_o = (got.cpu().numpy() - base) / dt, (ref_o.cpu().numpy() - base) / dt
        assert rel_err(inc, inc_o) < 2e-5
    assert rel_err((p_sym.cpu().numpy() - px) / dt, zpx) < 2e-5
    assert rel_err((q_sym.cpu().numpy() - pa) / dt, zpa) < 2e-5


def test_sharded_matching_nccl_single_rank():
    """SecondOrderSurfaceMatching with options['processGroup'] (the sharded rows, gathers and FP64 all-reduce on
    NCCL, world size 1) gives the same objective and gradient as the unsharded driver."""
    import os
    import torch
    import torch.distributed as dist
    from base.kernelFunctions import Kernel
    from base.surfaceMatching import SecondOrderSurfaceMatching
    from base.surfaces import Surface
    from base.syntheticShapes import icosphere, bumpy_ellipsoid
    x0, F = icosphere(3)
    x1 = bumpy_ellipsoid(x0, seed=0)
    a0 = np.random.default_rng(10).normal(0, 0.02, x0.shape)

    def make(pg):
        K = Kernel(name='gauss', sigma=0.5)
        K.pk_dtype = 'float32'
        opts = dict(maxIter=2, affine='none', KparDiff=K, KparDist=('gauss', 0.3), errorType='varifold',
                    pk_dtype='float32', timeStep=0.1, verb=False, initialMomentum=a0, processGroup=pg)
        return SecondOrderSurfaceMatching(Template=Surface(surf=(F, x0)), Target=Surface(surf=(F, x1)), options=opts)

    os.environ.setdefault('MASTER_ADDR', '127.0.0.1')
    os.environ.setdefault('MASTER_PORT', str(29900 + os.getpid() % 90))
    dist.init_process_group('nccl', rank=0, world_size=1)
    try:
        fs = make(True)
        obj_s = fs.objectiveFun()
        g_s = fs.getGradient(1.0)['a0'].clone()
        fs.optimizeMatching()
        torch.cuda.synchronize()
    finally:
        dist.destroy_process_group()
    fu = make(None)
    obj_u = fu.objectiveFun()
    g_u = fu.getGradient(1.0)['a0']
    fu.optimizeMatching()
    # At world size 1 the shooting and adjoint steps run the same (whole-step) kernels in both drivers; the kinetic
    # term K(x0)a0 does not: the sharded driver sums its row range, the unsharded one evaluates the self-sum once per
    # unordered pair. Both are FP32 compensated sums, so they agree to FP32 rounding, not bit for bit.
    assert abs(obj_s - obj_u) <= 1e-9 * abs(obj_u)
    assert rel_err(g_s.cpu().numpy(), g_u.cpu().numpy()) < 1e-6
    assert abs(fs.history[-1] - fu.history[-1]) <= 1e-7 * abs(fu.history[-1])
