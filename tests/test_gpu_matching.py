"""End-to-end parity of the device-resident matching drivers with the reference's own runs
(tests/golden/matching_*_L2.npz: SurfaceMatching / SecondOrderSurfaceMatching, level-2 icosphere -> bumpy
ellipsoid, Gaussian or Laplacian (order 3) deformation kernel sigma 0.5, varifold sigma 0.3, T = 10, BFGS,
5 iterations, float64).

FP64 path: objective at iteration 0 and first gradient within 1e-10, objective after every iteration within 1e-7
(the same BFGS / weak-Wolfe decisions). FP32 compensated path: objective 1e-6, gradient 2e-5, per-iteration
objectives 1e-4.
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN, rel_err

pytestmark = pytest.mark.gpu


def _options(dtype, maxIter, family='gauss'):
    from base.kernelFunctions import Kernel
    K = Kernel(name='laplacian', sigma=0.5, order=3) if family == 'laplacian' else Kernel(name='gauss', sigma=0.5)
    return dict(mode='normal', maxIter=maxIter, affine='none', regWeight=1.0, KparDiff=K,
                KparDist=('gauss', 0.3), sigmaError=1.0, errorType='varifold', pk_dtype=dtype, algorithm='bfgs',
                timeStep=0.1, verb=False)


@pytest.mark.parametrize('family', ['gauss', 'laplacian'])
@pytest.mark.parametrize('order', ['first', 'second'])
@pytest.mark.parametrize('dtype', ['float64', 'float32'])
def test_matching_vs_reference(order, dtype, family):
    """Gaussian deformation kernel, or the Laplacian kernel of order 3 (fixtures matching_*_lap_L2)."""
    from base.surfaceMatching import SurfaceMatching, SecondOrderSurfaceMatching
    from base.surfaces import Surface
    tag = '_lap' if family == 'laplacian' else ''
    d = np.load(os.path.join(GOLDEN, f'matching_{order}{tag}_L2.npz'))
    F = d['faces']
    cls = SurfaceMatching if order == 'first' else SecondOrderSurfaceMatching
    f = cls(Template=Surface(surf=(F, d['x0'])), Target=Surface(surf=(F, d['x1'])),
            options=_options(dtype, 5, family))
    t_obj, t_grad, t_it = (1e-10, 1e-10, 1e-7) if dtype == 'float64' else (1e-6, 2e-5, 1e-4)
    obj0 = f.objectiveFun()
    assert abs(obj0 - float(d['obj0'])) < t_obj * abs(float(d['obj0']))
    key = 'at' if order == 'first' else 'a0'
    g0 = f.getGradient(f.gradCoeff)[key].cpu().numpy()
    assert rel_err(g0, d['grad0']) < t_grad
    f.optimizeMatching()
    objs = np.array(f.history)
    ref = d['objs']
    assert objs.shape == ref.shape, (objs, ref)
    assert np.max(np.abs(objs - ref) / np.abs(ref)) < t_it, (objs, ref)
    if dtype == 'float64':
        assert rel_err(f.control[key].cpu().numpy(), d['control']) < 1e-6


def test_matching_gradient_matches_central_differences():
    """The optimiser's gradient against central FD of the objective along random directions (the reference's own
    TestGradient probe, base/bfgs.py:167-176), on the FP64 path."""
    import torch
    from base.surfaceMatching import SecondOrderSurfaceMatching
    from base.surfaces import Surface
    from base.syntheticShapes import icosphere, bumpy_ellipsoid
    x0, F = icosphere(3)
    x1 = bumpy_ellipsoid(x0, seed=0)
    f = SecondOrderSurfaceMatching(Template=Surface(surf=(F, x0)), Target=Surface(surf=(F, x1)),
                                   options=_options('float64', 3))
    f.control['a0'] = torch.from_numpy(np.random.default_rng(0).normal(0, 0.01, x0.shape)).cuda()
    f.obj = None
    f.objectiveFun()
    g = f.getGradient(1.0)
    torch.manual_seed(0)
    for _ in range(3):
        v = f.randomDir()
        h = 1e-6
        fp = f.updateTry(v, -h)
        fm = f.updateTry(v, h)
        fd = (fp - fm) / (2 * h)
        an = f.dotProduct_euclidean(g, [v])[0]
        assert abs(fd - an) < 1e-6 * max(1.0, abs(an)), (fd, an)
