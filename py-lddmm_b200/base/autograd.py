"""torch.autograd Functions over the hand-written shooting / data-term adjoint kernels.

* `GeodesicShooting.apply(x0, a0, K, timeStep, checkpoint_every)` -> (x_T, a_T): second-order shooting
  (base/pointEvolution.py:385-472). Backward = the reference's adjoint sweep (secondOrderCovector,
  base/pointEvolution.py:489-552), which is the transposed Jacobian of the Euler scheme: with (p_x, p_a) at T set to
  the incoming gradients, (p_x, p_a) at 0 are the gradients with respect to (x0, a0). Only every
  `checkpoint_every`-th state is kept in the forward pass; each segment is recomputed from its checkpoint during
  the backward sweep (memory O(T/k + k) states instead of O(T)).
* `LandmarkShooting.apply(x0, at, K, checkpoint_every)` -> x_T: first-order shooting (base/pointEvolution.py:88)
  with the sym transposed-Jacobian sweep (landmarkHamiltonianCovector with regweight 0) and dL/da_t = dt K(x_t) p_{t+1}.
* `SurfaceData.apply(xdef, term)` -> |S_def - S_1|^2 (varifold / current / measure, base/surfaceDistances.py) with
  the fused gradient kernel as backward.
* `Kinetic.apply(x, a, K)` -> 0.5 a.K(x)a with grad_a = K(x)a and grad_x = DK^T(x; a, a).

All tensors are float64 CUDA tensors; every sum runs in the sm_100a library.
"""
import numpy as np
import torch

from . import _native as nat
from . import pointEvolution as evol


def _sigma(K):
    s = np.asarray(K.sigma, dtype=float).ravel()
    if s.size != 1:
        raise NotImplementedError('the autograd Functions use one kernel width')
    K._check()
    return float(s[0])


def _step_forward(K, x, a, dt, origin, ws):
    x1, a1 = torch.empty_like(x), torch.empty_like(a)
    nat.check(nat.lib().lddmm_second_order_step(nat.ptr(x), nat.ptr(a), x.shape[0], _sigma(K), K.code, float(dt),
                                                origin, nat.ptr(x1), nat.ptr(a1), K.precision, ws[0], ws[1],
                                                nat.stream_ptr()), 'second_order_step')
    return x1, a1


def _step_adjoint(K, x, a, px, pa, dt, origin, ws):
    px0, pa0 = torch.empty_like(px), torch.empty_like(pa)
    nat.check(nat.lib().lddmm_second_order_adjoint_step(nat.ptr(x), nat.ptr(a), nat.ptr(px), nat.ptr(pa), x.shape[0],
                                                        _sigma(K), K.code, float(dt), origin, nat.ptr(px0),
                                                        nat.ptr(pa0), K.precision, ws[0], ws[1], nat.stream_ptr()),
              'second_order_adjoint_step')
    return px0, pa0


class GeodesicShooting(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x0, a0, K, timeStep, checkpoint_every=5):
        T = int(np.round(1.0 / timeStep))
        k = max(1, int(checkpoint_every))
        x0, a0 = x0.detach().contiguous(), a0.detach().contiguous()
        origin_list = nat.centroid(x0)
        origin = nat.origin_arg(origin_list)
        ws = nat.workspace(x0.shape[0], x0.shape[0], K.precision)
        checkpoints = [(x0, a0)]
        x, a = x0, a0
        for t in range(T):
            x, a = _step_forward(K, x, a, timeStep, origin, ws)
            if (t + 1) % k == 0 and t + 1 < T:
                checkpoints.append((x, a))
        ctx.K, ctx.dt, ctx.T, ctx.k, ctx.origin = K, timeStep, T, k, origin_list
        ctx.checkpoints = checkpoints
        return x, a

    @staticmethod
    def backward(ctx, gx, ga):
        K, dt, T, k = ctx.K, ctx.dt, ctx.T, ctx.k
        origin = nat.origin_arg(ctx.origin)
        x0 = ctx.checkpoints[0][0]
        ws = nat.workspace(x0.shape[0], x0.shape[0], K.precision)
        px = torch.zeros_like(x0) if gx is None else gx.contiguous().to(torch.float64)
        pa = torch.zeros_like(x0) if ga is None else ga.contiguous().to(torch.float64)
        n_seg = len(ctx.checkpoints)
        for s in range(n_seg - 1, -1, -1):
            t0 = s * k
            t1 = min(T, t0 + k)
            # recompute the states t0 .. t1-1 of this segment from its checkpoint
            x, a = ctx.checkpoints[s]
            states = [(x, a)]
            for _ in range(t0, t1 - 1):
                x, a = _step_forward(K, x, a, dt, origin, ws)
                states.append((x, a))
            for x, a in reversed(states):
                px, pa = _step_adjoint(K, x, a, px, pa, dt, origin, ws)
        ctx.checkpoints = None
        return px, pa, None, None, None


class LandmarkShooting(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x0, at, K, checkpoint_every=5):
        x0, at = x0.detach().contiguous(), at.detach().contiguous()
        xt = evol.shoot_first_order(x0, at, K)
        ctx.save_for_backward(xt, at)
        ctx.K = K
        return xt[-1].clone()

    @staticmethod
    def backward(ctx, gx):
        xt, at = ctx.saved_tensors
        T = at.shape[0]
        pxt, dat = evol.first_order_gradient(xt, at, gx.contiguous().to(torch.float64), ctx.K, 0.0, euclidean=True)
        # dat_t = K(x_t)(0 - p_{t+1}) = -K(x_t) p_{t+1};  dL/da_t = dt K(x_t) p_{t+1}
        return pxt[0], -dat / T, None, None


class SurfaceData(torch.autograd.Function):
    @staticmethod
    def forward(ctx, xdef, term, with_norm0=True):
        xdef = xdef.detach().contiguous()
        e = term.energy(xdef, with_norm0=with_norm0)
        ctx.term = term
        ctx.save_for_backward(xdef)
        return e[0] + e[1]

    @staticmethod
    def backward(ctx, g):
        (xdef,) = ctx.saved_tensors
        return ctx.term.gradient(xdef) * g, None, None


class Kinetic(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, a, K):
        x, a = x.detach().contiguous(), a.detach().contiguous()
        ka = K.applyK(x, a)
        ctx.save_for_backward(x, a, ka)
        ctx.K = K
        return 0.5 * (a * ka).sum()

    @staticmethod
    def backward(ctx, g):
        x, a, ka = ctx.saved_tensors
        gx = ctx.K.applyDiffKT(x, a, a) if ctx.needs_input_grad[0] else None
        return (None if gx is None else gx * g), ka * g, None


def geodesic_registration_loss(x0, a0, K, term, timeStep, sigmaError=1.0, checkpoint_every=5):
    """0.5 a0.K(x0)a0 + |S(x_T) - S_1|^2 / sigmaError^2, the objective of SecondOrderSurfaceMatching
    (base/secondOrderPointSetMatching.py:113-148 + base/surfaceMatching.py:443-466), differentiable in a0 and x0."""
    xT, _ = GeodesicShooting.apply(x0, a0, K, timeStep, checkpoint_every)
    return Kinetic.apply(x0, a0, K) + SurfaceData.apply(xT, term) / sigmaError ** 2
