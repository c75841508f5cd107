"""The L-BFGS search direction in one library call (lddmm_lbfgs_direction) against the optimiser's own two-loop
recursion (base/bfgs.py), on random pairs and inside a registration."""
import ctypes

import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu


def _two_loop(g, S, Y):
    """The recursion of base/bfgs.py:183-198 in float64 numpy."""
    q = g.copy()
    rho, alpha = [], []
    for s, y in reversed(list(zip(S, Y))):
        rho.append(1.0 / (y @ s))
        alpha.append(rho[-1] * (s @ q))
        q = q - alpha[-1] * y
    rho.reverse()
    alpha.reverse()
    c = (S[-1] @ Y[-1]) / (Y[-1] @ Y[-1])
    c = 1.0 if c < 1e-10 else c
    q = q * c
    for k in range(len(S)):
        beta = rho[k] * (Y[k] @ q)
        q = q + (alpha[k] - beta) * S[k]
    return q


@pytest.mark.parametrize('m,n', [(1, 7686), (7, 30726), (50, 7686), (64, 1000), (3, 1)])
def test_fused_direction_matches_two_loop(m, n):
    import torch
    from base import _native as nat
    rng = np.random.default_rng(m * 100 + n % 97)
    S = [rng.normal(size=n) for _ in range(m)]
    Y = [s + 0.3 * rng.normal(size=n) for s in S]          # positive curvature pairs, as BFGS keeps
    g = rng.normal(size=n)
    St = [torch.from_numpy(s).cuda() for s in S]
    Yt = [torch.from_numpy(y).cuda() for y in Y]
    gt = torch.from_numpy(g).cuda()
    q = torch.empty_like(gt)
    sp = (ctypes.c_void_p * m)(*[t.data_ptr() for t in St])
    yp = (ctypes.c_void_p * m)(*[t.data_ptr() for t in Yt])
    rc = nat.lib().lddmm_lbfgs_direction(ctypes.cast(sp, ctypes.c_void_p), ctypes.cast(yp, ctypes.c_void_p), m,
                                         nat.ptr(gt), n, nat.ptr(q), nat.stream_ptr())
    assert rc == 0
    assert rel_err(q.cpu().numpy(), _two_loop(g, S, Y)) < 1e-12
    q2 = torch.empty_like(gt)
    nat.lib().lddmm_lbfgs_direction(ctypes.cast(sp, ctypes.c_void_p), ctypes.cast(yp, ctypes.c_void_p), m,
                                    nat.ptr(gt), n, nat.ptr(q2), nat.stream_ptr())
    assert torch.equal(q, q2)                                 # fixed reduction order: bitwise reproducible


@pytest.mark.parametrize('dtype', ['float64', 'float32'])
def test_registration_with_fused_direction(dtype):
    """A level-3 registration (30 BFGS iterations) with the fused direction and with the optimiser's own recursion:
    the same iterates (objective histories within 1e-10 relative in FP64, 1e-4 in FP32)."""
    from base.kernelFunctions import Kernel
    from base.surfaceMatching import SecondOrderSurfaceMatching
    from base.surfaces import Surface
    from base.syntheticShapes import icosphere, bumpy_ellipsoid
    x0, F = icosphere(3)
    x1 = bumpy_ellipsoid(x0, seed=4)

    def run(fused):
        K = Kernel(name='gauss', sigma=0.5)
        K.pk_dtype = dtype
        opts = dict(maxIter=30, affine='none', regWeight=1.0, KparDiff=K, KparDist=('gauss', 0.3), sigmaError=1.0,
                    errorType='varifold', pk_dtype=dtype, algorithm='bfgs', timeStep=0.1, verb=False)
        f = SecondOrderSurfaceMatching(Template=Surface(surf=(F, x0)), Target=Surface(surf=(F, x1)), options=opts)
        if not fused:
            f.LBFGS_FUSED_MAX = 0
        f.optimizeMatching()
        return np.array(f.history)

    a, b = run(True), run(False)
    assert a.shape == b.shape and a.shape[0] >= 10
    tol = 1e-10 if dtype == 'float64' else 1e-4
    assert np.max(np.abs(a - b) / np.abs(b)) < tol
