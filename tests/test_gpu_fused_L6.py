"""Level-6 checks of the fused kernels, in the forms level 6 runs them (Gaussian FP32: the second-order forward step
and the varifold gradient in their expanded-distance forms, the adjoint step in the difference form), against the
FP64 oracle on 2,048 sampled target rows.

Problem of the level-6 registration: icosphere level 6 (40,962 vertices, 81,920 faces), deformation widths 0.25 and
0.5, varifold width 0.2, T = 20 (dt = 0.05). Momenta are smoothed (K_0.3 of N(0, 0.1^2)), covectors are the
varifold gradient at the deformed surface (px) and a smoothed field (pa), so every sum has the scale it has in a
registration. The step increments (x1 - x)/dt and (a1 - a)/dt are compared, not x1 itself, whose x part would hide
the error of the sums.
"""
import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu

TOL = 2e-5      # relative L2 error of shooting steps and gradients (FP32 compensated path)
DT = 0.05


@pytest.fixture(scope='module')
def level6():
    import oracle as O
    from base.syntheticShapes import icosphere, bumpy_ellipsoid
    x, F = icosphere(6)
    x1 = bumpy_ellipsoid(x, seed=0)
    rng = np.random.default_rng(5)
    a = O.apply_k(x, x, rng.normal(0, 0.1, x.shape), 0.3)
    a *= 0.3 / np.linalg.norm(O.apply_k(x, x, a, 0.5), axis=1).max()
    pa = O.apply_k(x, x, rng.normal(0, 0.1, x.shape), 0.3)
    xdef = x + 0.5 * O.apply_k(x, x, a, 0.5)
    rows = np.sort(rng.choice(x.shape[0], 2048, replace=False))
    return dict(x=x, F=F, x1=x1, a=a, pa=pa, xdef=xdef, rows=rows)


def _varifold_covector(d):
    """px = -(varifold gradient at the deformed surface), the end-point covector of a registration (FP64 path)."""
    if 'px' not in d:
        from base.kernelFunctions import Kernel
        from base.surfaceDistances import SurfaceDataTerm
        Kd = Kernel(name='gauss', sigma=0.2)
        Kd.pk_dtype = 'float64'
        term = SurfaceDataTerm(d['F'], d['x1'], d['F'], Kd, kind='varifold')
        d['px'] = -term.gradient(d['xdef']).cpu().numpy()
    return d['px']


def _run_step(nat, torch, X, A, sigma, precision):
    n = X.shape[0]
    x1, a1 = torch.empty_like(X), torch.empty_like(X)
    ws, wsb = nat.workspace(n, n, precision)
    nat.check(nat.lib().lddmm_second_order_step(nat.ptr(X), nat.ptr(A), n, sigma, nat.KERNEL_GAUSS, DT,
                                                nat.origin_arg(nat.centroid(X)), nat.ptr(x1), nat.ptr(a1), precision,
                                                ws, wsb, nat.stream_ptr()), 'second_order_step')
    return ((x1 - X) / DT).cpu().numpy(), ((a1 - A) / DT).cpu().numpy()


def _run_adjoint(nat, torch, X, A, PX, PA, sigma, precision):
    n = X.shape[0]
    px0, pa0 = torch.empty_like(X), torch.empty_like(X)
    ws, wsb = nat.workspace(n, n, precision)
    nat.check(nat.lib().lddmm_second_order_adjoint_step(nat.ptr(X), nat.ptr(A), nat.ptr(PX), nat.ptr(PA), n, sigma,
                                                        nat.KERNEL_GAUSS, DT, nat.origin_arg(nat.centroid(X)),
                                                        nat.ptr(px0), nat.ptr(pa0), precision, ws, wsb,
                                                        nat.stream_ptr()), 'second_order_adjoint_step')
    return ((px0 - PX) / DT).cpu().numpy(), ((pa0 - PA) / DT).cpu().numpy()


@pytest.mark.parametrize('sigma', [0.25, 0.5])
def test_second_order_step_level6(level6, sigma):
    import torch
    import oracle as O
    from base import _native as nat
    d = level6
    X, A = torch.from_numpy(d['x']).cuda(), torch.from_numpy(d['a']).cuda()
    zx, za = _run_step(nat, torch, X, A, sigma, nat.FP32C)
    rx, ra = O.second_order_step_rows(d['x'], d['a'], d['rows'], sigma)
    assert rel_err(zx[d['rows']], rx) < TOL
    assert rel_err(za[d['rows']], ra) < TOL


@pytest.mark.parametrize('sigma', [0.25, 0.5])
def test_second_order_adjoint_step_level6(level6, sigma):
    import torch
    import oracle as O
    from base import _native as nat
    d = level6
    px = _varifold_covector(d)
    X, A = torch.from_numpy(d['x']).cuda(), torch.from_numpy(d['a']).cuda()
    PX, PA = torch.from_numpy(px).cuda(), torch.from_numpy(d['pa']).cuda()
    zpx, zpa = _run_adjoint(nat, torch, X, A, PX, PA, sigma, nat.FP32C)
    rpx, rpa = O.second_order_adjoint_step_rows(d['x'], d['a'], px, d['pa'], d['rows'], sigma)
    assert rel_err(zpx[d['rows']], rpx) < TOL
    assert rel_err(zpa[d['rows']], rpa) < TOL


def test_varifold_gradient_level6(level6):
    import oracle as O
    from base.kernelFunctions import Kernel
    from base.surfaceDistances import SurfaceDataTerm
    d = level6
    Kd = Kernel(name='gauss', sigma=0.2)
    Kd.pk_dtype = 'float32'
    term = SurfaceDataTerm(d['F'], d['x1'], d['F'], Kd, kind='varifold')
    got = term.gradient(d['xdef']).cpu().numpy()
    ref = O.varifold_norm_gradient_rows(d['xdef'], d['F'], d['x1'], d['F'], 0.2, d['rows'])
    assert rel_err(got[d['rows']], ref) < TOL
