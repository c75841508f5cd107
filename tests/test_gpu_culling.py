"""Kernel widths small against the shape, and the exact culling of far face tiles in the surface data terms.

With a width small against the shape, tile pairs of a mesh stored in a spatially coherent order can be farther
apart than the distance at which exp underflows to exactly zero (FP32: 2^-126 flushed; FP64: below exp(-745)); the
varifold / current / measure kernels skip them. The varifold test below uses such a width (sigma 0.05 on the unit
sphere: most face-tile pairs are culled) against the float64 oracle, which evaluates every pair. The other tests
run the deformation-kernel sums at such widths (every tile evaluated there), against the oracle and against the
same sums over a shuffled copy of the points.

Tolerances (relative L2 error against float64): FP32 compensated path 2e-5, FP64 path 1e-12.
"""
import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu


def kernel(sigma, dtype, name='gauss'):
    from base.kernelFunctions import Kernel
    K = Kernel(name=name, sigma=sigma)
    K.pk_dtype = dtype
    return K


@pytest.mark.parametrize('dtype,sigma', [('float32', 0.05), ('float64', 0.02)])
def test_culled_kernel_sums_match_the_oracle(dtype, sigma):
    import oracle as O
    from base.syntheticShapes import icosphere
    x, _ = icosphere(5)
    rng = np.random.default_rng(11)
    a, p = rng.normal(size=x.shape), rng.normal(size=x.shape)
    K = kernel(sigma, dtype)
    tol = 2e-5 if dtype == 'float32' else 1e-12
    assert rel_err(K.applyK(x, a), O.apply_k(x, x, a, sigma)) < tol
    assert rel_err(K.applyDiffKT(x, p, a, sym=True), O.apply_diff_kt(x, x, p, a, sigma, sym=True)) < tol
    assert rel_err(K.applyDDiffK11and12(x, a, a, p), O.apply_ddiff_k11and12(x, a, a, p, sigma)) < tol
    # the same sums over shuffled points: no tile pair is far apart, every pair is evaluated
    perm = rng.permutation(x.shape[0])
    inv = np.argsort(perm)
    assert rel_err(K.applyK(x[perm], a[perm])[inv], K.applyK(x, a)) < tol


def test_culled_shooting_and_laplacian_match_the_oracle():
    import oracle as O
    from base import pointEvolution as evol
    from base.syntheticShapes import icosphere, smooth_momenta
    x0, _ = icosphere(4)
    rng = np.random.default_rng(12)
    a0 = smooth_momenta(x0, rng, O.apply_k, sigma_smooth=0.06, sigma_def=0.05, vmax=0.05)
    px1 = rng.normal(0, 0.5, x0.shape)
    g = evol.secondOrderGradient(x0, a0, px1, np.zeros_like(x0), kernel(0.05, 'float32'), 0.25)
    ref = O.second_order_gradient(x0, a0, px1, np.zeros_like(x0), 0.05, 0.25)
    errs = {k: rel_err(g[k], ref[k]) for k in ('xt', 'at', 'da0', 'pxt', 'pat')}
    assert all(e < 2e-5 for e in errs.values()), errs
    # Laplacian: exp(-r/sigma) reaches zero only beyond 127 sigma / log2(e) in FP32; at sigma 0.005 that is 0.44
    a = rng.normal(size=x0.shape)
    KL = kernel(0.005, 'float32', 'laplacian')
    assert rel_err(KL.applyK(x0, a), O.laplacian.apply_k(x0, x0, a, 0.005, 3)) < 2e-5


@pytest.mark.parametrize('level,sigma', [(4, 0.05), (5, 0.1)])
def test_culled_varifold_matches_the_oracle(level, sigma):
    """Level 4 at sigma 0.05: face blocks too wide for the expanded-distance energy kernel (difference form);
    level 5 at sigma 0.1: expanded form, with the tile pairs farther apart than 1.3 culled."""
    import oracle as O
    from base.surfaceDistances import SurfaceDataTerm
    from base.syntheticShapes import icosphere, bumpy_ellipsoid
    x0, F = icosphere(level)
    x1 = bumpy_ellipsoid(x0, seed=0)
    Kd = kernel(sigma, 'float32')
    term = SurfaceDataTerm(F, x1, F, Kd, kind='varifold')
    e = float(term.energy(x0)[0])
    e_ref = O.varifold_norm_def(x0, F, x1, F, sigma)
    assert abs(e - e_ref) < 1e-6 * abs(e_ref)
    g = term.gradient(x0).cpu().numpy()
    assert rel_err(g, O.varifold_norm_gradient(x0, F, x1, F, sigma)) < 2e-5
