"""Adjoint check (config: level-5 icosphere, smoothed random momenta, T = 20 geodesic shooting, varifold sigma 0.2,
checkpointing every 5 steps): the torch.autograd gradient of the registration objective against central finite
differences (h = 1e-4, 32 random directions, FP64 path) and against the reference's float64 gradient (the oracle's
secondOrderGradient with the varifold end-point gradient, base/pointEvolution.py:555-618)."""
import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu


def _setup(level, dtype):
    import torch
    import oracle as O
    from base.kernelFunctions import Kernel
    from base.surfaceDistances import SurfaceDataTerm
    from base.syntheticShapes import icosphere, bumpy_ellipsoid, smooth_momenta
    x0, F = icosphere(level)
    x1 = bumpy_ellipsoid(x0, seed=0)
    a0 = smooth_momenta(x0, np.random.default_rng(1), O.apply_k, sigma_smooth=0.3, sigma_def=0.5, vmax=0.2)
    K = Kernel(name='gauss', sigma=0.5)
    K.pk_dtype = dtype
    Kd = Kernel(name='gauss', sigma=0.2)
    Kd.pk_dtype = dtype
    term = SurfaceDataTerm(F, x1, F, Kd, kind='varifold')
    X0 = torch.from_numpy(x0).cuda()
    A0 = torch.from_numpy(a0).cuda()
    return x0, F, x1, a0, K, term, X0, A0


def test_autograd_vs_central_fd_l5():
    import torch
    from base.autograd import geodesic_registration_loss
    x0, F, x1, a0, K, term, X0, A0 = _setup(5, 'float64')
    A = A0.clone().requires_grad_(True)
    loss = geodesic_registration_loss(X0, A, K, term, 0.05, checkpoint_every=5)
    loss.backward()
    g = A.grad.detach()
    gen = torch.Generator(device='cuda').manual_seed(0)
    h = 1e-4
    worst = 0.0
    with torch.no_grad():
        for _ in range(32):
            v = torch.randn(A0.shape, generator=gen, dtype=torch.float64, device='cuda')
            v /= v.norm()
            fp = float(geodesic_registration_loss(X0, A0 + h * v, K, term, 0.05))
            fm = float(geodesic_registration_loss(X0, A0 - h * v, K, term, 0.05))
            fd = (fp - fm) / (2 * h)
            an = float((g * v).sum())
            worst = max(worst, abs(fd - an) / max(abs(an), 1e-3 * float(g.norm())))
    assert worst < 1e-5, worst


def test_checkpointing_is_exact_and_fp32_close():
    import torch
    from base.autograd import geodesic_registration_loss
    x0, F, x1, a0, K, term, X0, A0 = _setup(4, 'float64')
    grads = {}
    for k in (1, 5, 7, 20):
        A = A0.clone().requires_grad_(True)
        geodesic_registration_loss(X0, A, K, term, 0.05, checkpoint_every=k).backward()
        grads[k] = A.grad.detach()
    for k in (5, 7, 20):
        assert torch.equal(grads[k], grads[1]), k     # recomputation replays the same kernels: bitwise equal
    _, _, _, _, K32, term32, _, _ = _setup(4, 'float32')
    A = A0.clone().requires_grad_(True)
    geodesic_registration_loss(X0, A, K32, term32, 0.05, checkpoint_every=5).backward()
    assert rel_err(A.grad.cpu().numpy(), grads[1].cpu().numpy()) < 2e-5


def test_autograd_vs_reference_gradient_l5():
    import oracle as O
    import torch
    from base.autograd import geodesic_registration_loss
    x0, F, x1, a0, K, term, X0, A0 = _setup(5, 'float32')
    A = A0.clone().requires_grad_(True)
    geodesic_registration_loss(X0, A, K, term, 0.05, checkpoint_every=5).backward()
    xt, at = O.second_order_evolution(x0, a0, 0.5, 0.05)
    px1 = -O.varifold_norm_gradient(xt[-1], F, x1, F, 0.2)
    ref = O.second_order_gradient(x0, a0, px1, np.zeros_like(x0), 0.5, 0.05)['da0']
    assert rel_err(A.grad.cpu().numpy(), ref) < 2e-5


def test_first_order_and_data_autograd():
    """LandmarkShooting and SurfaceData against central FD on a level-3 problem (FP64 path)."""
    import torch
    from base.autograd import LandmarkShooting, SurfaceData
    from base.kernelFunctions import Kernel
    from base.surfaceDistances import SurfaceDataTerm
    from base.syntheticShapes import icosphere, bumpy_ellipsoid
    x0, F = icosphere(3)
    x1 = bumpy_ellipsoid(x0, seed=0)
    K = Kernel(name='gauss', sigma=0.5)
    K.pk_dtype = 'float64'
    Kd = Kernel(name='gauss', sigma=0.3)
    Kd.pk_dtype = 'float64'
    term = SurfaceDataTerm(F, x1, F, Kd)
    X0 = torch.from_numpy(x0).cuda()
    at = torch.from_numpy(np.random.default_rng(2).normal(0, 0.002, (10,) + x0.shape)).cuda()
    A = at.clone().requires_grad_(True)
    X = X0.clone().requires_grad_(True)
    loss = SurfaceData.apply(LandmarkShooting.apply(X, A, K), term)
    loss.backward()
    h = 1e-6
    for which, base, grad in (('a', at, A.grad), ('x', X0, X.grad)):
        v = torch.randn(base.shape, dtype=torch.float64, device='cuda')
        with torch.no_grad():
            if which == 'a':
                f = lambda s: float(SurfaceData.apply(LandmarkShooting.apply(X0, at + s * v, K), term))
            else:
                f = lambda s: float(SurfaceData.apply(LandmarkShooting.apply(X0 + s * v, at, K), term))
            fd = (f(h) - f(-h)) / (2 * h)
        an = float((grad * v).sum())
        assert abs(fd - an) < 1e-5 * max(1.0, abs(an)), (which, fd, an)
