"""Learned momentum proposal: the BF16 tensor-core GEMM in every layout, the network's forward / backward kernels
against a float64 CPU restatement (oracle/learned.py), the nearest-target feature, and what a trained network gains
over the plain optimiser started from zero momentum.

Tolerances: FP32-output GEMMs 1e-5 relative (bf16 inputs are exact in FP32; only the summation order differs),
BF16-output GEMMs 1e-2 (one bf16 rounding); network gradients 3e-2 relative (bf16 activations and deltas).
"""
import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu


def _gemm(ta, tb, epi, A, B, M, N, K, bias=None, mask=None, splits=1):
    import torch
    from base import _native as nat
    out_dtype = torch.float32 if epi in (0, 1) else torch.bfloat16
    C = torch.empty((M, N), dtype=out_dtype, device='cuda')
    ws = torch.empty(splits * M * N, dtype=torch.float32, device='cuda') if splits > 1 else None
    nat.check(nat.lib().lddmm_bf16_gemm(ta, tb, epi, M, N, K, nat.ptr(A), nat.ptr(B), nat.ptr(bias), nat.ptr(mask),
                                        nat.ptr(C), splits, nat.ptr(ws), 0 if ws is None else ws.numel() * 4,
                                        nat.stream_ptr()))
    return C


@pytest.mark.parametrize('ta', [0, 1])
@pytest.mark.parametrize('tb', [0, 1])
def test_bf16_gemm_layouts_and_epilogues(ta, tb):
    import torch
    M, N, K = 192, 128, 96
    g = torch.Generator(device='cuda').manual_seed(ta * 2 + tb)
    A = torch.randn((M, K), generator=g, device='cuda').to(torch.bfloat16)
    B = torch.randn((K, N), generator=g, device='cuda').to(torch.bfloat16)
    bias = torch.randn(N, generator=g, device='cuda')
    As = A.t().contiguous() if ta else A
    Bs = B.t().contiguous() if tb else B
    ref = A.float() @ B.float()
    assert rel_err(_gemm(ta, tb, 0, As, Bs, M, N, K).cpu(), ref.cpu()) < 1e-5
    assert rel_err(_gemm(ta, tb, 1, As, Bs, M, N, K, bias=bias).cpu(), (ref + bias).cpu()) < 1e-5
    r = _gemm(ta, tb, 2, As, Bs, M, N, K, bias=bias).float()
    assert rel_err(r.cpu(), torch.relu(ref + bias).cpu()) < 1e-2
    mask = torch.relu(torch.randn((M, N), generator=g, device='cuda')).to(torch.bfloat16)
    r = _gemm(ta, tb, 4, As, Bs, M, N, K, mask=mask).float()
    assert rel_err(r.cpu(), (ref * (mask.float() > 0)).cpu()) < 1e-2


def test_gemm_split_k_is_deterministic():
    import torch
    M, N, K = 128, 128, 64 * 97
    g = torch.Generator(device='cuda').manual_seed(7)
    At = torch.randn((K, M), generator=g, device='cuda').to(torch.bfloat16)
    B = torch.randn((K, N), generator=g, device='cuda').to(torch.bfloat16)
    one = _gemm(1, 0, 0, At, B, M, N, K)
    s8 = _gemm(1, 0, 0, At, B, M, N, K, splits=8)
    assert rel_err(s8.cpu(), one.cpu()) < 1e-5
    assert torch.equal(_gemm(1, 0, 0, At, B, M, N, K, splits=8), s8)
    assert rel_err(one.cpu(), (At.float().t() @ B.float()).cpu()) < 1e-5


def test_network_gradients_vs_cpu_oracle():
    """Device gradients against the oracle with the same bf16 storage points (1e-2) and against exact arithmetic
    (8e-2: three layers of bf16 deltas and activations)."""
    import torch
    from oracle.learned import mlp_loss_and_grads, mlp_loss_and_grads_bf16
    from base.learnedProposal import MomentumProposal, IN_DIM, N_FEATURES, N_OUT
    model = MomentumProposal(seed=3)
    M = 1024
    g = torch.Generator(device='cuda').manual_seed(1)
    F = torch.zeros((M, IN_DIM), device='cuda')
    F[:, :N_FEATURES] = torch.randn((M, N_FEATURES), generator=g, device='cuda')
    F = F.to(torch.bfloat16)
    T = torch.randn((M, N_OUT), generator=g, device='cuda')
    for i in range(4):          # non-trivial biases so that every term of the backward pass is exercised
        model.b[i].normal_(0.0, 0.1)
    model.Wb = [w.to(torch.bfloat16) for w in model.W]
    loss, grads = model.gradients(F, T, M, weight=1.0 / M)
    Wb = [w.float() for w in model.Wb]
    for oracle_fn, tol in ((mlp_loss_and_grads_bf16, 1e-2), (mlp_loss_and_grads, 8e-2)):
        ref_loss, _, ref = oracle_fn(F.float(), Wb, model.b, T, N_OUT, 1.0 / M)
        assert abs(float(loss) - float(ref_loss)) < tol * float(ref_loss)
        for k, (a, r) in enumerate(zip(grads, ref)):
            if float(r.norm()) == 0.0:
                assert float(a.norm()) == 0.0
                continue
            assert rel_err(a.cpu().double().numpy(), r.numpy()) < tol, (oracle_fn.__name__, k)


def test_nearest_displacement():
    import torch
    from base.learnedProposal import nearest_displacement
    rng = np.random.default_rng(0)
    x = rng.normal(size=(777, 3))
    y = rng.normal(size=(1300, 3))
    d = nearest_displacement(torch.from_numpy(x).cuda(), torch.from_numpy(y).cuda()).cpu().numpy()
    idx = ((x[:, None, :] - y[None, :, :]) ** 2).sum(-1).argmin(axis=1)
    assert np.allclose(d, y[idx] - x, atol=1e-12)


def test_trained_proposal_beats_zero_momentum():
    """Train on 384 pairs generated by shooting (level-3 sphere), then on held-out pairs: the proposal lowers the
    registration objective below the zero-momentum start, and BFGS from the warm start reaches the plain run's
    final objective in fewer iterations."""
    import torch
    from base import learnedProposal as lp
    from base.surfaceMatching import SecondOrderSurfaceMatching
    from base.surfaces import Surface
    from base.syntheticShapes import icosphere
    from base.kernelFunctions import Kernel
    x0, F = icosphere(3)
    feats, labels, _, n = lp.generate_pairs(x0, F, 384, seed=0, timeStep=0.1)
    model = lp.MomentumProposal(seed=0)
    hist = lp.train(model, feats, labels, n, epochs=40, batch_pairs=16, lr=2e-3)
    assert hist[-1] < 0.2 * hist[0], hist
    # held-out pairs: fresh momenta (seed 123); their targets are shot again below
    feats_h, labels_h, momenta_h, _ = lp.generate_pairs(x0, F, 4, seed=123, timeStep=0.1)
    with torch.no_grad():
        y = model.forward(feats_h.reshape(-1, lp.IN_DIM)).reshape(4, -1, lp.OUT_DIM)[:, :n, :3]
    label_err = float((y - labels_h[:, :n]).norm() / labels_h[:, :n].norm())
    assert label_err < 0.3, label_err   # held-out momentum-density error
    gains = []
    for i in range(4):
        a_true = momenta_h[i]
        K = Kernel(name='gauss', sigma=0.5)
        K.pk_dtype = 'float32'
        from base import pointEvolution as evol
        X0 = torch.from_numpy(x0).cuda()
        xt, _ = evol.shoot_second_order(X0, a_true, K, 0.1)
        x1 = xt[-1].cpu().numpy()
        opts = dict(maxIter=25, affine='none', regWeight=1.0, KparDiff=K, KparDist=('gauss', 0.3), sigmaError=0.1,
                    errorType='varifold', pk_dtype='float32', algorithm='bfgs', timeStep=0.1, verb=False)
        plain = SecondOrderSurfaceMatching(Template=Surface(surf=(F, x0)), Target=Surface(surf=(F, x1)),
                                           options=dict(opts))
        plain.optimizeMatching()
        warm = SecondOrderSurfaceMatching(Template=Surface(surf=(F, x0)), Target=Surface(surf=(F, x1)),
                                          options=dict(opts))
        used, obj_prop, obj_zero, _ = lp.warm_start(warm, model)
        assert used and obj_prop < 0.5 * obj_zero, (obj_prop, obj_zero)
        warm.optimizeMatching()
        target = plain.history[-1]
        it_plain = next(k for k, v in enumerate(plain.history) if v <= target * (1 + 1e-9))
        it_warm = next((k for k, v in enumerate(warm.history) if v <= target * (1 + 1e-9)), len(warm.history))
        gains.append((it_plain, it_warm))
    assert sum(w for _, w in gains) < sum(p for p, _ in gains), gains


def test_prolong_momentum_keeps_the_velocity_field():
    """A smooth momentum on the level-3 sphere carried to the level-4 sphere generates the same velocity field at the
    fine points (0.37% relative L2 in a float64 numpy emulation of the same formula; the bound leaves room for the
    FP32 kernel sums)."""
    import torch
    from base import learnedProposal as lp
    from base.kernelFunctions import Kernel
    from base.syntheticShapes import icosphere
    xc, Fc = icosphere(3)
    xf, _ = icosphere(4)
    rng = np.random.default_rng(0)
    K = Kernel(name='gauss', sigma=0.5)
    K.pk_dtype = 'float64'
    Ks = Kernel(name='gauss', sigma=0.4)
    Ks.pk_dtype = 'float64'
    ac = Ks.applyK(xc, rng.normal(size=xc.shape))
    af = lp.prolong_momentum(xc, ac, xf, K, 0.4 * lp.mean_edge_length(xc, Fc))
    v_coarse = K.applyK(xc, ac, firstVar=xf)
    v_fine = K.applyK(torch.from_numpy(xf).cuda(), af).cpu().numpy()
    assert rel_err(v_fine, v_coarse) < 1e-2


def test_multilevel_warm_start_reaches_the_plain_optimum_sooner():
    """Coarse-to-fine warm start (network at the coarsest level, plain BFGS at levels 2 and 3, prolongation to level
    4) on a bumpy-ellipsoid registration: the fine level takes the prolonged momentum, whose objective is far below
    the zero-momentum start, and BFGS from it reaches the plain run's final objective in fewer fine iterations."""
    import torch  # noqa: F401
    from base import learnedProposal as lp
    from base.kernelFunctions import Kernel
    from base.surfaceMatching import SecondOrderSurfaceMatching
    from base.surfaces import Surface
    from base.syntheticShapes import icosphere, bumpy_ellipsoid
    x0, F = icosphere(4)
    x1 = bumpy_ellipsoid(x0, seed=3)
    xs, Fs = icosphere(2)
    feats, labels, _, n = lp.generate_pairs(xs, Fs, 128, seed=0, timeStep=0.1)
    model = lp.MomentumProposal(seed=0)
    lp.train(model, feats, labels, n, epochs=20, batch_pairs=16, lr=2e-3)

    def matching(maxIter=60):
        K = Kernel(name='gauss', sigma=0.5)
        K.pk_dtype = 'float32'
        opts = dict(maxIter=maxIter, affine='none', regWeight=1.0, KparDiff=K, KparDist=('gauss', 0.3),
                    sigmaError=1.0, errorType='varifold', pk_dtype='float32', algorithm='bfgs', timeStep=0.1,
                    verb=False)
        return SecondOrderSurfaceMatching(Template=Surface(surf=(F, x0)), Target=Surface(surf=(F, x1)),
                                          options=opts)

    plain = matching()
    obj_zero = plain.objectiveFun()
    plain.optimizeMatching()
    target = plain.history[-1]
    warm = matching()
    rec = lp.multilevel_warm_start(warm, model, [icosphere(2)[::-1], icosphere(3)[::-1]], rtol=1e-4)
    assert [lv['vertices'] for lv in rec['levels']] == [162, 642]
    assert rec['prolonged_used'] and rec['obj_prolonged'] < 0.2 * obj_zero, rec
    warm.optimizeMatching()
    it_plain = next(k for k, v in enumerate(plain.history) if v <= target * (1 + 1e-9))
    it_warm = next((k for k, v in enumerate(warm.history) if v <= target * (1 + 1e-9)), len(warm.history))
    assert it_warm < it_plain, (it_warm, it_plain)
    # the same warm start through the options of the matching class: the same start and the same iterates
    via = matching()
    via.options['warmStart'] = {'model': model, 'coarse': [icosphere(2)[::-1], icosphere(3)[::-1]], 'rtol': 1e-4}
    via.optimizeMatching()
    got, want = via.warmStartRecord['levels'], rec['levels']
    assert [lv['iters'] for lv in got] == [lv['iters'] for lv in want]
    # the vertex normals of the features are summed with atomic adds: agreement to rounding, not bitwise
    assert np.allclose([lv['objective'] for lv in got], [lv['objective'] for lv in want], rtol=1e-9, atol=0)
    assert len(via.history) == len(warm.history)
    assert np.allclose(via.history, warm.history, rtol=1e-6, atol=0)


def test_shapes_law_pairs():
    """The 'shapes' momentum law (quadratic stretch + bumps + smoothed noise along the normals): momenta are normal
    fields, their initial speeds lie in [vmin, vmax], the labels are the momentum densities, and the draw is
    reproducible from the seed (to rounding)."""
    import torch
    from base import learnedProposal as lp
    from base.kernelFunctions import Kernel
    from base.syntheticShapes import icosphere
    x0, F = icosphere(3)
    feats, labels, momenta, n = lp.generate_pairs(x0, F, 8, seed=5, timeStep=0.1, law='shapes', vmin=0.1, vmax=0.3)
    X0 = torch.from_numpy(x0).cuda()
    nrm = lp.vertex_normals(X0, torch.from_numpy(F).cuda())
    K = Kernel(name='gauss', sigma=0.5)
    K.pk_dtype = 'float64'
    mass = lp.kernel_mass(K, X0)
    for i in range(8):
        a = momenta[i]
        tangential = a - (a * nrm).sum(dim=1, keepdim=True) * nrm
        assert float(tangential.norm()) < 1e-9 * float(a.norm())
        v = K.applyK(X0, a).norm(dim=1).max()
        assert 0.1 * (1 - 1e-5) <= float(v) <= 0.3 * (1 + 1e-5)   # speeds set with the FP32 kernel sum
        assert rel_err(labels[i, :n].double().cpu().numpy(), (a * mass / lp.MOMENTUM_SCALE).cpu().numpy()) < 1e-6
    # the vertex normals are accumulated with atomic adds (index_add_), so a second draw agrees to rounding
    _, _, again, _ = lp.generate_pairs(x0, F, 8, seed=5, timeStep=0.1, law='shapes', vmin=0.1, vmax=0.3)
    assert rel_err(again.cpu().numpy(), momenta.cpu().numpy()) < 1e-12


def test_generate_pairs_graph_replay_matches_eager():
    """The CUDA-graph replay of a pair's pipeline (speed rescale, shooting, features, label) gives the eager path's
    features, labels and momenta (to the rounding of the atomically summed vertex normals)."""
    from base import learnedProposal as lp
    from base.syntheticShapes import icosphere
    x0, F = icosphere(3)
    out = {g: lp.generate_pairs(x0, F, 6, seed=9, timeStep=0.1, law='shapes', graph=g) for g in (True, False)}
    (fg, lg, mg, _), (fe, le, me, _) = out[True], out[False]
    assert rel_err(mg.cpu().numpy(), me.cpu().numpy()) < 1e-12
    assert rel_err(lg.double().cpu().numpy(), le.double().cpu().numpy()) < 1e-6
    assert rel_err(fg.float().cpu().numpy(), fe.float().cpu().numpy()) < 1e-2     # bf16 features
