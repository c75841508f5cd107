"""Parity of the Laplacian (Matern) kernel family with the reference: KernelSpec(name='laplacian', order=q),
K(r) = P_q(r/sigma) exp(-r/sigma) (base/kernelFunctions_util.py:20-56, lap_fun* functors).

Fixtures: outputs of the reference's own float64 numba path (tests/golden/laplacian_*.npz). Larger sizes: the CPU
oracle (oracle/laplacian.py, pinned to those fixtures in test_oracle_golden.py).

Tolerances (relative L2 error of the output array against float64): FP32 compensated path 3e-5 on the random-sign
fixture inputs, 2e-5 for shooting and its adjoint; FP64 path 1e-12 (operators), 1e-10 (shooting adjoint).
"""
import glob
import os

import numpy as np
import pytest

from conftest import GOLDEN, rel_err

pytestmark = pytest.mark.gpu

LFILES = sorted(glob.glob(os.path.join(GOLDEN, 'laplacian_L2_o*.npz')))
TOL_OPS = {'float32': 3e-5, 'float64': 1e-12}
TOL_SHOOT = {'float32': 2e-5, 'float64': 1e-10}


def kernel(sigma, order, dtype):
    from base.kernelFunctions import Kernel
    K = Kernel(name='laplacian', sigma=sigma, order=order)
    K.pk_dtype = dtype
    return K


@pytest.mark.parametrize('dtype', ['float32', 'float64'])
@pytest.mark.parametrize('path', LFILES, ids=os.path.basename)
def test_laplacian_operators_vs_reference(path, dtype):
    d = np.load(path)
    K = kernel(float(d['sigma']), int(d['order']), dtype)
    x, y, a, p, q = d['x'], d['y'], d['a'], d['p'], d['q']
    ny = y.shape[0]
    checks = {
        'applyK': K.applyK(x, a),
        'applyK_cross': K.applyK(x, a, firstVar=y),
        'applyDiffKT': K.applyDiffKT(x, p, a),
        'applyDiffKT_cross': K.applyDiffKT(x, p[:ny], a, firstVar=y),
        'applyDiffKT_sym': K.applyDiffKT(x, p, a, sym=True),
        'applyDiffKT_lddmm': K.applyDiffKT(x, p, a, lddmm=True, regweight=float(d['regweight'])),
        'applyDDiffK11and12': K.applyDDiffK11and12(x, a, q, p),
        'applyDiffK1and2': K.applyDiffK1and2(x, p, a),
        'applyDivergence': K.applyDivergence(x, a),
    }
    errs = {k: rel_err(v, d[k]) for k, v in checks.items()}
    bad = {k: e for k, e in errs.items() if not e < TOL_OPS[dtype]}
    assert not bad, (os.path.basename(path), dtype, bad)


@pytest.mark.parametrize('dtype', ['float32', 'float64'])
def test_laplacian_shooting_vs_reference(dtype):
    from base import pointEvolution as evol
    d = np.load(os.path.join(GOLDEN, 'laplacian_shooting_L2_o3.npz'))
    K = kernel(float(d['sigma']), int(d['order']), dtype)
    tol = TOL_SHOOT[dtype]
    st = evol.landmarkDirectEvolutionEuler(d['x0'], d['at'], K)
    assert rel_err(st['xt'], d['fo_xt']) < tol
    dat, _, pxt = evol.landmarkHamiltonianGradient(d['x0'], d['at'], d['px1'], K, float(d['regweight']),
                                                   getCovector=True)
    assert rel_err(dat, d['fo_dat']) < tol
    assert rel_err(pxt, d['fo_pxt']) < tol
    g = evol.secondOrderGradient(d['x0'], d['a0'], d['px1'], d['pa1'], K, float(d['timeStep']))
    want = {'xt': d['xt'], 'at': d['at_so'], 'da0': d['da0'], 'pxt': d['pxt'], 'pat': d['pat']}
    errs = {k: rel_err(g[k], v) for k, v in want.items()}
    assert all(e < tol for e in errs.values()), errs


@pytest.mark.parametrize('order', [0, 2, 3])
def test_laplacian_l4_vs_oracle(order):
    """Level 4 (2,562 points), smooth momenta: applyK / applyDiffKT(sym) / applyDDiffK11and12 / applyDiffK1and2
    and the second-order adjoint in FP32 against the oracle (orders without a reference fixture included)."""
    import oracle as O
    from base import pointEvolution as evol
    from base.syntheticShapes import icosphere, smooth_momenta
    L = O.laplacian
    x0, _ = icosphere(4)
    rng = np.random.default_rng(17 + order)
    a = smooth_momenta(x0, rng, O.apply_k, sigma_smooth=0.4, sigma_def=0.5, vmax=0.3)
    p = smooth_momenta(x0, rng, O.apply_k, sigma_smooth=0.3, sigma_def=0.5, vmax=0.5)
    K = kernel(0.4, order, 'float32')
    assert rel_err(K.applyK(x0, a), L.apply_k(x0, x0, a, 0.4, order)) < 5e-6
    assert rel_err(K.applyDiffKT(x0, p, a, sym=True), L.apply_diff_kt(x0, x0, p, a, 0.4, sym=True, order=order)) \
        < 2e-5
    if order >= 2:   # the second-derivative table is zero below order 2 (as in the reference)
        assert rel_err(K.applyDDiffK11and12(x0, a, a, p), L.apply_ddiff_k11and12(x0, a, a, p, 0.4, order)) < 2e-5
    assert rel_err(K.applyDiffK1and2(x0, p, a), L.apply_diff_k1and2(x0, p, a, 0.4, order)) < 2e-5
    px1 = rng.normal(0, 0.5, x0.shape)
    ref = O.second_order_gradient(x0, a, px1, np.zeros_like(x0), 0.4, 0.2, L.ops(order))
    g = evol.secondOrderGradient(x0, a, px1, np.zeros_like(x0), K, 0.2)
    errs = {k: rel_err(g[k], ref[k]) for k in ('xt', 'at', 'da0', 'pxt', 'pat')}
    assert all(e < 2e-5 for e in errs.values()), errs


@pytest.mark.parametrize('order', [1, 3])
def test_laplacian_first_order_l4_vs_oracle(order):
    """First-order shooting and adjoint with the Laplacian kernel at level 4 (several row blocks of the symmetric
    adjoint step), FP32 against the oracle: trajectory, covectors and the gradient (relative L2 2e-5)."""
    import torch
    import oracle as O
    from base import pointEvolution as evol
    from base.syntheticShapes import icosphere
    L = O.laplacian
    x0, _ = icosphere(4)
    rng = np.random.default_rng(31 + order)
    T, w = 4, 0.7
    at = np.stack([O.apply_k(x0, x0, rng.normal(0, 0.02, x0.shape), 0.3) for _ in range(T)])
    px1 = rng.normal(size=x0.shape)
    K = kernel(0.4, order, 'float32')
    AT = torch.from_numpy(at).cuda()
    xt = evol.shoot_first_order(torch.from_numpy(x0).cuda(), AT, K, regweight=w)
    dat_ref, xt_ref, pxt_ref = O.landmark_hamiltonian_gradient(x0, at, px1, 0.4, w, L.ops(order))
    assert rel_err(xt.cpu().numpy() - x0, xt_ref - x0) < 2e-5
    pxt, dat = evol.first_order_gradient(xt, AT, torch.from_numpy(px1).cuda(), K, w)
    assert rel_err(pxt.cpu().numpy() - px1, pxt_ref - px1) < 2e-5
    assert rel_err(dat.cpu().numpy(), dat_ref) < 2e-5


def test_laplacian_multiscale_and_dense_matrix():
    """Two widths weighted sigma^-1 / sum sigma^-1 (base/kernelFunctions_util.py:451-466) and getK."""
    import oracle as O
    from base.kernelFunctions import Kernel
    from base.syntheticShapes import icosphere
    x, _ = icosphere(3)
    rng = np.random.default_rng(3)
    a = rng.normal(size=x.shape)
    K = Kernel(name='laplacian', sigma=[0.3, 0.6], order=3)
    K.pk_dtype = 'float64'
    w = np.array([0.3, 0.6]) ** -1.0
    w /= w.sum()
    want = w[0] * O.laplacian.apply_k(x, x, a, 0.3, 3) + w[1] * O.laplacian.apply_k(x, x, a, 0.6, 3)
    assert rel_err(K.applyK(x, a), want) < 1e-12
    G = K.getK(x)
    assert rel_err(G @ a, want) < 1e-12


def test_laplacian_is_rejected_where_not_implemented():
    from base.kernelFunctions import Kernel
    from base.surfaceDistances import SurfaceDataTerm
    from base.syntheticShapes import icosphere
    x, F = icosphere(1)
    K = Kernel(name='laplacian', sigma=0.5)
    with pytest.raises(NotImplementedError):
        K.applyKTensor(x, np.ones(len(x)), np.ones(len(x)), x, x)
    with pytest.raises(NotImplementedError):
        SurfaceDataTerm(F, x, F, K, kind='varifold')
