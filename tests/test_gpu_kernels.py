"""Parity of the CUDA kernel operators (through the C-ABI, via the drop-in `Kernel`) with the reference.

Fixtures: outputs of the reference's own float64 numba path (tests/golden). Larger sizes: the CPU oracle
(pinned to the reference in test_oracle_golden.py). Full size (L6): size-independent properties.

Tolerances (relative L2 error of the output array against float64):
  FP32 compensated path ('float32'): 2e-5 for random-sign momenta fixtures (cancellation), 5e-6 for smooth momenta;
  FP64 path ('float64'): 1e-12.
"""
import glob
import os

import numpy as np
import pytest

from conftest import GOLDEN, rel_err

pytestmark = pytest.mark.gpu

KFILES = sorted(glob.glob(os.path.join(GOLDEN, 'kernels_*.npz')))
TOL = {'float32': 2e-5, 'float64': 1e-12}


def kernel(sigma, dtype):
    from base.kernelFunctions import Kernel
    K = Kernel(name='gauss', sigma=sigma)
    K.pk_dtype = dtype
    return K


@pytest.mark.parametrize('dtype', ['float32', 'float64'])
@pytest.mark.parametrize('path', KFILES, ids=os.path.basename)
def test_kernel_operators_vs_reference(path, dtype):
    d = np.load(path)
    K = kernel(float(d['sigma']), dtype)
    x, y, a, p, q = d['x'], d['y'], d['a'], d['p'], d['q']
    ny = y.shape[0]
    tol = TOL[dtype]
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
        'applyDivergence_cross': K.applyDivergence(x, a, firstVar=y),
        'applyKTensor': K.applyKTensor(x, d['ay'], d['ay'], d['betay'], d['betay']),
        'applyKTensor_cross': K.applyKTensor(x, d['ay'][:ny], d['ay'], d['betay'][:ny], d['betay'], firstVar=y),
    }
    if 'beta' in d:
        checks['applyDiffKmat'] = K.applyDiffKmat(x, d['beta'])
        checks['applyK_mat'] = K.applyK(x, d['u'], matrixWeights=True)
    errs = {k: rel_err(v, d[k]) for k, v in checks.items()}
    for k, v in checks.items():
        assert isinstance(v, np.ndarray) and v.dtype == np.float64 and v.shape == d[k].shape, k
    dense_tol = 1e-12  # dense-weight kernels always run in FP64
    bad = {k: e for k, e in errs.items() if e > (dense_tol if k in ('applyDiffKmat', 'applyK_mat') else tol)}
    assert not bad, f'{dtype}: {bad}'


@pytest.mark.parametrize('dtype', ['float32', 'float64'])
def test_apply_k_larger_vs_oracle(dtype):
    import oracle as O
    from base.syntheticShapes import icosphere
    x, _ = icosphere(4)
    rng = np.random.default_rng(0)
    a = O.apply_k(x, x, rng.normal(0, 0.1, x.shape), 0.3)      # smooth momenta
    for sigma in (0.25, 0.5):
        K = kernel(sigma, dtype)
        ref = O.apply_k(x, x, a, sigma)
        tol = 5e-6 if dtype == 'float32' else 1e-12
        assert rel_err(K.applyK(x, a), ref) < tol
        assert rel_err(K.applyDiffKT(x, a, a), O.apply_diff_kt(x, x, a, a, sigma)) < tol
        assert rel_err(K.applyDDiffK11and12(x, a, a, a * 0.5 + 0.1),
                       O.apply_ddiff_k11and12(x, a, a, a * 0.5 + 0.1, sigma)) < 4 * tol


def test_expanded_and_difference_forms_agree():
    """applyK's FP32 kernel evaluates a target block in the expanded-distance form when the block is small in
    kernel widths and in the difference form otherwise. Level 6 at sigma 0.15: the icosphere's own point order gives
    compact blocks (mostly expanded), a shuffled copy blocks spanning the sphere (difference form); the two must
    agree with each other and with the oracle (on 2,048 sampled targets). Sigma 1.0 puts the shuffled blocks in the
    expanded form as well."""
    import oracle as O
    from base.syntheticShapes import icosphere
    x, _ = icosphere(6)
    rng = np.random.default_rng(3)
    a = rng.normal(0, 0.1, x.shape)
    perm = rng.permutation(x.shape[0])
    inv = np.argsort(perm)
    rows = rng.choice(x.shape[0], 2048, replace=False)
    for sigma in (0.15, 1.0):
        K = kernel(sigma, 'float32')
        ref = O.apply_k(x[rows], x, a, sigma)
        ordered = K.applyK(x, a)
        shuffled = K.applyK(x[perm], a[perm])[inv]
        assert rel_err(ordered[rows], ref) < 5e-6, sigma
        assert rel_err(shuffled[rows], ref) < 5e-6, sigma
        assert rel_err(ordered, shuffled) < 5e-6, sigma


@pytest.mark.parametrize('n,m', [(1, 1), (1, 7), (7, 1), (33, 129), (129, 33), (511, 513), (1000, 0), (0, 10)])
def test_ragged_and_edge_sizes(n, m):
    import oracle as O
    rng = np.random.default_rng(n * 1000 + m)
    y = rng.normal(size=(n, 3))
    x = rng.normal(size=(m, 3))
    a = rng.normal(size=(m, 3))
    K = kernel(0.7, 'float32')
    out = K.applyK(x, a, firstVar=y)
    assert out.shape == (n, 3)
    if m == 0:
        assert np.all(out == 0)
    elif n > 0:
        assert rel_err(out, O.apply_k(y, x, a, 0.7)) < 2e-5
        p = rng.normal(size=(n, 3))
        assert rel_err(K.applyDiffKT(x, p, a, firstVar=y), O.apply_diff_kt(y, x, p, a, 0.7)) < 2e-5


@pytest.mark.parametrize('family', ['gauss', 'laplacian'])
@pytest.mark.parametrize('n', [1, 7, 511, 513, 1023, 1024, 1025, 2049, 5000])
@pytest.mark.parametrize('spread', ['ball', 'wide'])
def test_self_sum_ragged_sizes(n, spread, family):
    """K(x, x) a with one point array as targets and sources runs a symmetric kernel (each unordered pair once,
    credited to both points; Gaussian: 1,024 points per block, Laplacian: 512): sizes below, at and above one and
    two blocks, points in a small ball (Gaussian: expanded-distance form) or spread far in kernel widths (difference
    form for wide blocks), against the oracle and against the ordered-pair kernel (the same sum through a distinct
    target array)."""
    import oracle as O
    from base.kernelFunctions import Kernel
    rng = np.random.default_rng(n)
    scale = 0.5 if spread == 'ball' else 6.0
    x = rng.normal(size=(n, 3)) * scale
    a = rng.normal(size=(n, 3))
    if family == 'gauss':
        K = kernel(0.7, 'float32')
        ref = O.apply_k(x, x, a, 0.7)
    else:   # Laplacian of order 3: the difference-form symmetric kernel (row blocks of 512 points)
        K = Kernel(name='laplacian', sigma=0.7, order=3)
        K.pk_dtype = 'float32'
        ref = O.laplacian.apply_k(x, x, a, 0.7, 3)
    out = K.applyK(x, a)
    tol = 2e-5 if family == 'gauss' else 3e-5     # random-sign momenta: cancellation (Laplacian: its polynomial too)
    assert rel_err(out, ref) < tol
    assert rel_err(K.applyK(x, a, firstVar=x.copy()), ref) < tol


def test_full_size_properties_l6():
    """L6 (40,962 points): linearity, symmetry <b, K a> = <a, K b>, translation invariance and FP32 vs FP64."""
    import torch
    from base.syntheticShapes import icosphere
    x, _ = icosphere(6)
    rng = np.random.default_rng(1)
    X = torch.from_numpy(x).cuda()
    A = torch.from_numpy(rng.normal(size=x.shape)).cuda()
    B = torch.from_numpy(rng.normal(size=x.shape)).cuda()
    for sigma in (0.25, 0.5):
        K32, K64 = kernel(sigma, 'float32'), kernel(sigma, 'float64')
        ka, kb, kab = K32.applyK(X, A), K32.applyK(X, B), K32.applyK(X, A + B)
        assert rel_err((ka + kb).cpu(), kab.cpu()) < 2e-6
        s1, s2 = float((B * ka).sum()), float((A * kb).sum())
        assert abs(s1 - s2) < 1e-6 * (abs(s1) + abs(s2))
        shifted = K32.applyK(X + 3.0, A)
        assert rel_err(shifted.cpu(), ka.cpu()) < 2e-6
        k64 = K64.applyK(X, A)
        assert rel_err(ka.cpu(), k64.cpu()) < 2e-5


def test_multiscale_kernel_matches_weighted_sum():
    import oracle as O
    from base.syntheticShapes import icosphere
    from base.kernelFunctions import Kernel
    x, _ = icosphere(3)
    a = np.random.default_rng(2).normal(size=x.shape)
    K = Kernel(name='gauss', sigma=[0.25, 0.5])
    w = np.array([0.25, 0.5]) ** -1.0
    w /= w.sum()
    ref = w[0] * O.apply_k(x, x, a, 0.25) + w[1] * O.apply_k(x, x, a, 0.5)
    assert rel_err(K.applyK(x, a), ref) < 1e-12


def test_diffk_options_and_fd_probe():
    import oracle as O
    from base.syntheticShapes import icosphere
    x, _ = icosphere(2)
    rng = np.random.default_rng(4)
    a1, a2 = rng.normal(size=x.shape), rng.normal(size=x.shape)
    K = kernel(0.5, 'float64')
    both = K.applyDiffK1and2(x, a1, a2)
    assert rel_err(K.applyDiffK(x, a1, a2) + K.applyDiffK2(x, a1, a2), both) < 1e-12
    assert rel_err(both, O.apply_diff_k1and2(x, a1, a2, 0.5)) < 1e-12
    y = x[:50] * 1.1
    fd, an = K.testDiffKT(y, x, rng.normal(size=y.shape), a1)
    assert abs(fd - an) < 1e-5 * max(1.0, abs(an))


@pytest.mark.parametrize('dtype', ['float32', 'float64'])
def test_nan_propagates(dtype):
    """As in the reference (numpy arithmetic), a NaN coordinate or momentum reaches every sum it enters: a NaN source
    point or momentum makes every output NaN, a NaN target point only its own row (every exponential path, the
    FMA-pipe one included)."""
    from base.syntheticShapes import icosphere
    x, _ = icosphere(4)
    a = np.random.default_rng(4).normal(size=x.shape)
    K = kernel(0.5, dtype)
    xs = x.copy()
    xs[17, 1] = np.nan
    assert np.isnan(K.applyK(xs, a)).all()
    an = a.copy()
    an[5, 0] = np.nan
    assert np.isnan(K.applyK(x, an)[:, 0]).all()
    y = x[:1000].copy()
    y[::7, 2] = np.nan
    out = K.applyK(x, a, firstVar=y)
    assert np.isnan(out[::7]).all()
    rest = np.ones(y.shape[0], bool)
    rest[::7] = False
    assert np.isfinite(out[rest]).all()


def test_errors_are_loud():
    from base.kernelFunctions import Kernel
    from base._native import LddmmError
    K = Kernel(name='poly', sigma=0.5)      # a family the library does not implement
    with pytest.raises(NotImplementedError):
        K.applyK(np.zeros((4, 3)), np.zeros((4, 3)))
    import torch
    K = kernel(0.5, 'float32')
    Y = torch.zeros((4, 3), dtype=torch.float64, device='cuda')
    X = torch.zeros((5, 3), dtype=torch.float64, device='cuda')
    with pytest.raises(LddmmError):
        K._diff_kt(Y, X, Y, X, 1, 1.0)   # sym / lddmm need as many targets as sources: rejected by the library
