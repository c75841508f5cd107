"""Parity of the surface data-term kernels (varifold / current / measure) with the reference
(base/surfaceDistances.py). Tolerance (relative error against float64): FP32 compensated 2e-5 (energies 1e-6),
FP64 1e-11."""
import glob
import os

import numpy as np
import pytest

from conftest import GOLDEN, rel_err

pytestmark = pytest.mark.gpu
DFILES = sorted(glob.glob(os.path.join(GOLDEN, 'data_*.npz')))


def kernel(sigma, dtype):
    from base.kernelFunctions import Kernel
    K = Kernel(name='gauss', sigma=sigma)
    K.pk_dtype = dtype
    return K


@pytest.mark.parametrize('dtype', ['float32', 'float64'])
@pytest.mark.parametrize('path', DFILES, ids=os.path.basename)
def test_data_terms_vs_reference(path, dtype):
    from base import surfaceDistances as sd
    from base.surfaces import Surface
    d = np.load(path)
    K = kernel(float(d['sigma']), dtype)
    F = d['faces']
    fv1 = Surface(surf=(F, d['x1']))
    fvd = Surface(surf=(F, d['xdef']))
    fvw = Surface(surf=(F, d['xdef']), weights=d['weights'])
    te = 1e-6 if dtype == 'float32' else 1e-11
    tg = 2e-5 if dtype == 'float32' else 1e-11
    got = {
        'varifoldNorm0': (sd.varifoldNorm0(fv1, K), te),
        'varifoldNormDef': (sd.varifoldNormDef(fvd, fv1, K), te),
        'varifoldNormGradient': (sd.varifoldNormGradient(fvd, fv1, K), tg),
        'varifoldNormDef_w': (sd.varifoldNormDef(fvw, fv1, K), te),
        'varifoldNormGradient_w': (sd.varifoldNormGradient(fvw, fv1, K), tg),
        'currentNorm0': (sd.currentNorm0(fv1, K), te),
        'currentNormDef': (sd.currentNormDef(fvd, fv1, K), te),
        'currentNormGradient': (sd.currentNormGradient(fvd, fv1, K), tg),
        'measureNorm0': (sd.measureNorm0(fv1, K), te),
        'measureNormDef': (sd.measureNormDef(fvd, fv1, K), te),
        'measureNormGradient': (sd.measureNormGradient(fvd, fv1, K), tg),
    }
    bad = {k: rel_err(v, d[k]) for k, (v, t) in got.items() if rel_err(v, d[k]) > t}
    assert not bad, bad


def test_varifold_weight_gradient_vs_oracle():
    import oracle as O
    from base import surfaceDistances as sd
    from base.surfaces import Surface
    d = np.load(os.path.join(GOLDEN, 'data_L3_s0.2.npz'))
    F = d['faces']
    K = kernel(0.2, 'float64')
    fv1 = Surface(surf=(F, d['x1']))
    fvw = Surface(surf=(F, d['xdef']), weights=d['weights'])
    px, pxw = sd.varifoldNormGradient(fvw, fv1, K, with_weights=True)
    rpx, rpxw = O.varifold_norm_gradient(d['xdef'], F, d['x1'], F, 0.2, weights=d['weights'], with_weights=True)
    assert rel_err(px, rpx) < 1e-11 and rel_err(pxw, rpxw) < 1e-11


def test_varifold_l5_vs_oracle_and_fd():
    """L5 (20,480 faces), where the reference's dense gradient no longer fits: oracle + central FD on the GPU."""
    import torch
    import oracle as O
    from base.surfaceDistances import SurfaceDataTerm
    from base.syntheticShapes import icosphere, bumpy_ellipsoid
    x0, F = icosphere(5)
    x1 = bumpy_ellipsoid(x0, seed=0)
    xd = x0 * 1.05
    term = SurfaceDataTerm(F, x1, F, kernel(0.2, 'float32'), kind='varifold')
    g = term.gradient(xd).cpu().numpy()
    ref = O.varifold_norm_gradient(xd, F, x1, F, 0.2)
    assert rel_err(g, ref) < 2e-5
    e = float(term.energy(xd)[0])
    assert abs(e - O.varifold_norm_def(xd, F, x1, F, 0.2)) < 1e-6 * abs(e)
    term64 = SurfaceDataTerm(F, x1, F, kernel(0.2, 'float64'), kind='varifold')
    rng = np.random.default_rng(0)
    v = rng.normal(size=xd.shape)
    h = 1e-5
    fd = (float(term64.energy(xd + h * v)[0]) - float(term64.energy(xd - h * v)[0])) / (2 * h)
    an = float((term64.gradient(xd).cpu().numpy() * v).sum())
    assert abs(fd - an) < 1e-6 * abs(an)


def test_energy_is_deterministic():
    import torch
    from base.surfaceDistances import SurfaceDataTerm
    from base.syntheticShapes import icosphere, bumpy_ellipsoid
    x0, F = icosphere(4)
    x1 = bumpy_ellipsoid(x0, seed=0)
    term = SurfaceDataTerm(F, x1, F, kernel(0.3, 'float32'))
    e1 = term.energy(x0, with_norm0=True)
    g1 = term.gradient(x0)
    for _ in range(3):
        assert torch.equal(term.energy(x0, with_norm0=True), e1)
        assert torch.equal(term.gradient(x0), g1)
