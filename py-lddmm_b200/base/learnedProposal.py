"""Learned initial-momentum proposal for geodesic surface matching (no counterpart in the reference).

A per-vertex MLP maps local features of a (source, target) pair to the initial momentum a0 of
SecondOrderSurfaceMatching; the plain optimiser then refines from that proposal and falls back to zero momentum
when the proposal does not lower the objective (`warm_start`).

Features per source vertex (all computed on the device by the library's kernels):
  centred position (3), area-weighted vertex normal (3), nearest-target displacement d (3), its kernel-smoothed
  versions sum_l K(x_k,x_l) d_l / sum_l K(x_k,x_l) at widths 0.25 and 0.5 (6), normal component d.n (1), |d| (1),
  and the normalised kernel smoothings of d.n and |d| at widths 0.1, 0.2, 0.35 and 0.7 (8, the kernel-smoothed
  aggregation over the surface) -> 25, zero-padded to 64 (the GEMM tile width).
Network: 64 -> 128 -> 128 -> 128 -> 64 (outputs 0..2 used), ReLU, BF16 weights and activations, FP32 accumulation
and FP32 master weights (Adam), all GEMMs in `lddmm_bf16_gemm` (mma.sync tensor cores).
Output: the momentum density m = a0 * mass (N,3), mass_k = sum_l K(x_k, x_l) the kernel mass of the deformation
kernel, over MOMENTUM_SCALE. The density has velocity units and does not depend on the mesh resolution (the momentum
itself is a discrete measure that scales with 1/mass), so a network trained at one level applies at any other; the
proposal is a0 = m / mass. Predicting the momentum (a deconvolution of the displacement, which the multi-scale
features give the network) rather than the velocity K a0 matters: started from the exact normal velocity turned
into a momentum by the normalised kernel inverse, BFGS needs as many iterations as from the network's velocity,
three times more than from the exact momentum.

Training data: pairs generated by the method itself -- random smooth normal momentum fields shot with the
deformation kernel; the label is the momentum density of the generating momentum. Two laws for the scalar field
along the normals: 'noise' (a white-noise field smoothed by K_s, MOMENTUM_LAW) and 'shapes' (a mixture of a random
quadratic form, Gaussian bumps and the smoothed noise, MOMENTUM_LAW_SHAPES: the kinds of deformation a surface
registration meets); each is rescaled to an initial speed drawn in [vmin, vmax].

Coarse to fine (multilevel_warm_start): the proposal is made on a coarse triangulation of the source, refined there
by the plain optimiser, and its momentum density carried to the full-resolution source (prolong_momentum).
"""
import math

import numpy as np
import torch

from . import _native as nat
from . import pointEvolution as evol
from .kernelFunctions import Kernel

IN_DIM, HIDDEN, OUT_DIM, N_OUT = 64, 128, 64, 3
N_FEATURES = 25
MOMENTUM_SCALE = 0.3
# The law of the generating momenta of the training pairs (generate_pairs): normal fields, rescaled in speed. The
# unscaled law a = K_0.4 N(0, 0.3^2) per coordinate gives initial speeds of 7 to ~400 on the unit sphere (trajectories
# no registration produces), and its tangential part is invisible to the varifold data term (an ill-posed label).
MOMENTUM_LAW = ('a = (K_0.4 z) n: a scalar white-noise field z smoothed at width 0.4, along the vertex normals n, '
                'rescaled to a maximum initial speed drawn from U[0.05, 0.35]; shot with sigma 0.5, T = 10')
# The 'shapes' law: normal fields of the kinds of deformation a surface registration meets -- a random quadratic
# form (an ellipsoidal stretch: x^T M x with M a random symmetric matrix), a few Gaussian bumps (random centres on
# the surface, widths U[0.15, 0.45], signed heights) and the smoothed noise of MOMENTUM_LAW -- mixed with random
# weights and rescaled in speed like MOMENTUM_LAW.
MOMENTUM_LAW_SHAPES = ('a = (w1 q + w2 b + w3 K_0.4 z) n: q = x^T M x (M symmetric, N(0,1) entries), b = sum of '
                       'U{0..12} Gaussian bumps (centres on the surface, widths U[0.15, 0.45], heights N(0,1)), z '
                       'white noise, weights U[0,1], each field scaled to max 1; rescaled to a maximum initial speed '
                       'U[0.05, 0.35]; shot with sigma 0.5, T = 10')
SCALAR_WIDTHS = (0.1, 0.2, 0.35, 0.7)
# rows per split of the weight-gradient GEMMs (act^T dy, K = the batch's rows): split-K keeps the whole GPU busy
SPLIT_ROWS = 512
ROW_PAD = 64


def _pad_rows(n):
    return ((n + ROW_PAD - 1) // ROW_PAD) * ROW_PAD


def vertex_normals(X, faces_t):
    """Area-weighted vertex normals (sum of incident face surfels, normalised)."""
    v0, v1, v2 = X[faces_t[:, 0]], X[faces_t[:, 1]], X[faces_t[:, 2]]
    s = torch.cross(v1 - v0, v2 - v0, dim=1) * 0.5
    n = torch.zeros_like(X)
    for j in range(3):
        n.index_add_(0, faces_t[:, j], s)
    return n / n.norm(dim=1, keepdim=True).clamp_min(1e-12)


def nearest_displacement(X, Y):
    D = torch.empty_like(X)
    nat.check(nat.lib().lddmm_nearest_displacement(nat.ptr(X), X.shape[0], nat.ptr(Y), Y.shape[0], nat.ptr(D),
                                                   nat.stream_ptr()), 'nearest_displacement')
    return D


_SMOOTH = {}


def _smoother(sigma):
    K = _SMOOTH.get(sigma)
    if K is None:
        K = Kernel(name='gauss', sigma=sigma)
        K.pk_dtype = 'float32'
        _SMOOTH[sigma] = K
    return K


_MASSES = {}


def _smoother_mass(sigma, X0):
    """K_sigma(X0) 1 (N,3): the normaliser of the smoothed features, which depends on the source alone. Cached for
    the same source tensor object (the entry keeps a reference to it, so its memory cannot be reused by another
    array) while its in-place version counter is unchanged: pairs sharing a source compute it once."""
    e = _MASSES.get((sigma, id(X0)))
    if e is not None and e[0] is X0 and e[1] == X0._version:
        return e[2]
    if len(_MASSES) > 16:
        _MASSES.clear()
    m = _smoother(sigma).applyK(X0, torch.ones_like(X0))
    _MASSES[(sigma, id(X0))] = (X0, X0._version, m)
    return m


def pair_features(X0, faces_t, X1, normals=None):
    """(N, IN_DIM) bf16 feature matrix (rows padded to a multiple of 64 with zeros) for source X0 and target X1."""
    n = X0.shape[0]
    nrm = vertex_normals(X0, faces_t) if normals is None else normals
    d = nearest_displacement(X0, X1)
    dn = (d * nrm).sum(dim=1, keepdim=True)
    dl = d.norm(dim=1, keepdim=True)
    feats = [X0 - X0.mean(dim=0, keepdim=True), nrm, d]
    for s in (0.25, 0.5):
        feats.append(_smoother(s).applyK(X0, d) / _smoother_mass(s, X0))
    feats += [dn, dl]
    scal = torch.cat([dn, dl, torch.ones_like(dn)], dim=1).contiguous()   # one kernel sum smooths both and the mass
    for s in SCALAR_WIDTHS:
        r = _smoother(s).applyK(X0, scal)
        feats.append(r[:, :2] / r[:, 2:3])
    F = torch.zeros((_pad_rows(n), IN_DIM), dtype=torch.bfloat16, device=X0.device)
    F[:n, :N_FEATURES] = torch.cat(feats, dim=1).to(torch.bfloat16)
    return F


def kernel_mass(K, X):
    """mass_k = sum_l K(x_k, x_l) (N,1)."""
    return K.applyK(X, torch.ones_like(X))[:, :1]


class MomentumProposal:
    """Per-vertex MLP with hand-written BF16 forward / backward kernels and an Adam step kernel."""

    dims = (IN_DIM, HIDDEN, HIDDEN, HIDDEN, OUT_DIM)

    def __init__(self, seed=0, device='cuda'):
        g = torch.Generator(device='cpu').manual_seed(seed)
        self.W, self.b = [], []
        for i in range(4):
            fi, fo = self.dims[i], self.dims[i + 1]
            w = torch.randn((fi, fo), generator=g, dtype=torch.float32) * math.sqrt(2.0 / fi)
            if i == 0:
                w[N_FEATURES:] = 0.0
            if i == 3:
                w *= 0.1
                w[:, N_OUT:] = 0.0
            self.W.append(w.to(device))
            self.b.append(torch.zeros(fo, dtype=torch.float32, device=device))
        self.Wb = [w.to(torch.bfloat16) for w in self.W]
        self.m = [torch.zeros_like(t) for t in self.W + self.b]
        self.v = [torch.zeros_like(t) for t in self.W + self.b]
        self.step = 0

    # ------------------------------------------------------------------ kernels
    @staticmethod
    def _gemm(ta, tb, epi, A, B, C, M, N, K, bias=None, mask=None, splits=1, split_ws=None):
        sw, swb = (split_ws, split_ws.numel() * 4) if split_ws is not None else (None, 0)
        nat.check(nat.lib().lddmm_bf16_gemm(ta, tb, epi, M, N, K, nat.ptr(A), nat.ptr(B), nat.ptr(bias),
                                            nat.ptr(mask), nat.ptr(C), splits, nat.ptr(sw), swb, nat.stream_ptr()),
                  'bf16_gemm')

    def forward(self, F, keep=False):
        """F (M, IN_DIM) bf16, M a multiple of 64 -> (M, 64) f32 outputs (and the activations when keep)."""
        M = F.shape[0]
        acts = [F]
        h = F
        for i in range(3):
            out = torch.empty((M, self.dims[i + 1]), dtype=torch.bfloat16, device=F.device)
            self._gemm(0, 0, 2, h, self.Wb[i], out, M, self.dims[i + 1], self.dims[i], bias=self.b[i])
            acts.append(out)
            h = out
        y = torch.empty((M, OUT_DIM), dtype=torch.float32, device=F.device)
        self._gemm(0, 0, 1, h, self.Wb[3], y, M, OUT_DIM, HIDDEN, bias=self.b[3])
        return (y, acts) if keep else y

    def gradients(self, F, target, valid, weight=None):
        """Loss (device scalar) and FP32 gradients [dW0..dW3, db0..db3] of the mean squared error on the first 3
        outputs of rows < valid (target (M,3) f32)."""
        M = F.shape[0]
        y, acts = self.forward(F, keep=True)
        w = (1.0 / max(valid, 1)) if weight is None else weight
        dy = torch.empty((M, OUT_DIM), dtype=torch.bfloat16, device=F.device)
        row_loss = torch.empty(M, dtype=torch.float32, device=F.device)
        nat.check(nat.lib().lddmm_mse_grad(nat.ptr(y), M, OUT_DIM, nat.ptr(target), N_OUT, int(valid), float(w),
                                           nat.ptr(dy), nat.ptr(row_loss), nat.stream_ptr()), 'mse_grad')
        splits = max(1, min(64, M // SPLIT_ROWS))
        split_ws = torch.empty(splits * HIDDEN * HIDDEN, dtype=torch.float32, device=F.device) if splits > 1 else None
        col_ws = torch.empty(((M + 255) // 256) * max(self.dims), dtype=torch.float32, device=F.device)
        dW, db = [None] * 4, [None] * 4
        for i in range(3, -1, -1):
            fi, fo = self.dims[i], self.dims[i + 1]
            gw = torch.empty((fi, fo), dtype=torch.float32, device=F.device)
            sp = splits if split_ws is not None and fi * fo <= HIDDEN * HIDDEN else 1
            self._gemm(1, 0, 0, acts[i], dy, gw, fi, fo, M, splits=sp, split_ws=split_ws if sp > 1 else None)
            gb = torch.empty(fo, dtype=torch.float32, device=F.device)
            nat.check(nat.lib().lddmm_bf16_colsum(nat.ptr(dy), M, fo, nat.ptr(gb), nat.ptr(col_ws), col_ws.numel() * 4,
                                                  nat.stream_ptr()), 'colsum')
            dW[i], db[i] = gw, gb
            if i > 0:
                dx = torch.empty((M, fi), dtype=torch.bfloat16, device=F.device)
                self._gemm(0, 1, 4, dy, self.Wb[i], dx, M, fi, fo, mask=acts[i])
                dy = dx
        loss = row_loss.sum() * w
        return loss, dW + db

    def adam(self, grads, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8, weight_decay=0.0):
        self.step += 1
        params = self.W + self.b
        for k, (p, g) in enumerate(zip(params, grads)):
            pb = self.Wb[k] if k < 4 else None
            nat.check(nat.lib().lddmm_adam_step(nat.ptr(p), nat.ptr(g), nat.ptr(self.m[k]), nat.ptr(self.v[k]),
                                                nat.ptr(pb), p.numel(), lr, beta1, beta2, eps, self.step,
                                                weight_decay, nat.stream_ptr()), 'adam_step')

    # ------------------------------------------------------------------ inference
    def predict_density(self, X0, faces_t, X1, normals=None):
        """Predicted momentum density m = a0 * mass (N,3) f64 for registering X0 (with faces) onto X1."""
        n = X0.shape[0]
        F = pair_features(X0, faces_t, X1, normals)
        y = self.forward(F)
        return (y[:n, :N_OUT].to(torch.float64) * MOMENTUM_SCALE).contiguous()

    def predict(self, X0, faces_t, X1, Kdef, normals=None):
        """Initial momentum proposal a0 (N,3) f64: the predicted density divided by the kernel mass of Kdef."""
        return (self.predict_density(X0, faces_t, X1, normals) / kernel_mass(Kdef, X0)).contiguous()

    def state_dict(self):
        return {'W': [w.cpu() for w in self.W], 'b': [b.cpu() for b in self.b], 'step': self.step}

    def load_state_dict(self, d):
        self.W = [w.cuda() for w in d['W']]
        self.b = [b.cuda() for b in d['b']]
        self.Wb = [w.to(torch.bfloat16) for w in self.W]
        self.step = d.get('step', 0)


# ---------------------------------------------------------------------------------------------------------------
# Training data generated by the method itself, and training
# ---------------------------------------------------------------------------------------------------------------
def _shape_field(X0, gen, rng, Ksm):
    """One scalar field of the 'shapes' law (N,1): the quadratic form, the bumps and the smoothed noise, each scaled
    to max |.| = 1 and mixed with U[0,1] weights. Scalar parameters come from the host generator `rng` (no device
    synchronisation), the noise from the device generator `gen`."""
    n = X0.shape[0]
    dev, f64 = X0.device, torch.float64
    c = X0 - X0.mean(dim=0, keepdim=True)
    M = rng.normal(size=(3, 3))
    M = torch.from_numpy(0.5 * (M + M.T)).to(dev)
    q = ((c @ M) * c).sum(dim=1, keepdim=True)
    nb = int(rng.integers(0, 13))
    b = torch.zeros((n, 1), dtype=f64, device=dev)
    if nb:
        centres = X0[torch.from_numpy(rng.integers(0, n, nb)).to(dev)]                    # (nb, 3)
        w = torch.from_numpy(rng.uniform(0.15, 0.45, nb)).to(dev)
        h = torch.from_numpy(rng.normal(size=nb)).to(dev)
        d2 = ((X0[:, None, :] - centres[None, :, :]) ** 2).sum(dim=2)                    # (n, nb)
        b = (h[None, :] * torch.exp(-d2 / (2 * w[None, :] ** 2))).sum(dim=1, keepdim=True)
    z = torch.randn((n, 1), generator=gen, dtype=f64, device=dev).expand(n, 3).contiguous()
    zs = Ksm.applyK(X0, z)[:, :1]
    wts = rng.uniform(0.0, 1.0, 3)
    out = torch.zeros((n, 1), dtype=f64, device=dev)
    for wt, fld in zip(wts, (q, b, zs)):
        out = out + float(wt) * fld / fld.abs().max().clamp_min(1e-300)
    return out


def generate_pairs(x0, faces, n_pairs, seed=0, sigma_def=0.5, sigma_smooth=0.4, timeStep=0.1, vmin=0.05, vmax=0.35,
                   law='noise', graph=True):
    """Features (n_pairs, Mpad, IN_DIM) bf16, labels (n_pairs, Mpad, 3) f32 and momenta (n_pairs, n, 3) f64 of pairs
    (x0, shoot(x0, a_i)).

    a_i = (K_{sigma_smooth} z) n with z a scalar white-noise field, rescaled to an initial speed ~ U[vmin, vmax]
    (several widths: a sum of such fields, one per width, with random weights U[0, 1]);
    targets shot with K_{sigma_def} over round(1/timeStep) steps; labels are the momentum densities a_i * mass
    (mass of K_{sigma_def}), over MOMENTUM_SCALE. law='shapes' draws the scalar field from the law of
    MOMENTUM_LAW_SHAPES instead of smoothed noise alone.

    With `graph` the part of a pair after its random field -- the speed rescale, the shooting, the features and the
    label, ~30 launches of small level-4 kernels -- is captured once in a CUDA graph and replayed per pair (static
    input and output buffers), so the host issues one replay instead of the launches; the results are those of the
    eager path."""
    X0 = nat.as_device(x0)
    faces_t = torch.from_numpy(np.ascontiguousarray(faces, dtype=np.int64)).cuda()
    n = X0.shape[0]
    Mp = _pad_rows(n)
    Kdef = Kernel(name='gauss', sigma=sigma_def)
    Kdef.pk_dtype = 'float32'
    widths = tuple(sigma_smooth) if isinstance(sigma_smooth, (tuple, list)) else (sigma_smooth,)
    Ksm = []
    for w in widths:
        k = Kernel(name='gauss', sigma=w)
        k.pk_dtype = 'float32'
        Ksm.append(k)
    normals = vertex_normals(X0, faces_t)
    gen = torch.Generator(device='cuda').manual_seed(seed)
    speeds = torch.rand(n_pairs, generator=gen, dtype=torch.float64, device='cuda') * (vmax - vmin) + vmin
    feats = torch.zeros((n_pairs, Mp, IN_DIM), dtype=torch.bfloat16, device='cuda')
    labels = torch.zeros((n_pairs, Mp, N_OUT), dtype=torch.float32, device='cuda')
    momenta = torch.zeros((n_pairs, n, 3), dtype=torch.float64, device='cuda')
    origin = nat.centroid(X0)
    mass = kernel_mass(Kdef, X0)
    if law not in ('noise', 'shapes'):
        raise ValueError(f'unknown momentum law {law!r}')
    rng = np.random.default_rng(seed)

    def field():
        a = torch.zeros_like(X0)
        if law == 'shapes':
            a = _shape_field(X0, gen, rng, Ksm[0]) * normals
        for k in (Ksm if law == 'noise' else ()):
            z = torch.randn((n, 1), generator=gen, dtype=torch.float64, device='cuda').expand(n, 3).contiguous()
            f = k.applyK(X0, z)[:, :1]
            wt = torch.rand((), generator=gen, dtype=torch.float64, device='cuda') if len(Ksm) > 1 else 1.0
            a = a + wt * f / f.abs().max() * normals
        return a

    def finish(a_raw, speed):
        v = Kdef.applyK(X0, a_raw)
        a = a_raw * (speed / v.norm(dim=1).max())
        xt, _ = evol.shoot_second_order(X0, a, Kdef, timeStep, origin=origin)
        return a, pair_features(X0, faces_t, xt[-1], normals), (a * mass / MOMENTUM_SCALE).to(torch.float32)

    if graph and n_pairs > 1:
        a_in = torch.zeros_like(X0)
        s_in = torch.zeros((), dtype=torch.float64, device='cuda')
        a_in.copy_(normals)
        s_in.fill_(0.5 * (vmin + vmax))
        side = torch.cuda.Stream()
        side.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(side):      # warm-up: workspaces and cached normalisers exist before the capture
            for _ in range(2):
                finish(a_in, s_in)
        torch.cuda.current_stream().wait_stream(side)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            a_out, f_out, l_out = finish(a_in, s_in)
        for i in range(n_pairs):
            a_in.copy_(field())
            s_in.copy_(speeds[i])
            g.replay()
            feats[i] = f_out
            labels[i, :n] = l_out
            momenta[i] = a_out
        del g
        return feats, labels, momenta, n
    for i in range(n_pairs):
        a, f, lab = finish(field(), speeds[i])
        feats[i] = f
        labels[i, :n] = lab
        momenta[i] = a
    return feats, labels, momenta, n


def train(model, feats, labels, n, epochs=10, batch_pairs=16, lr=1e-3, seed=0, log=None):
    """Minibatch Adam on (n_pairs, Mp, .) tensors; returns the per-epoch mean training loss."""
    P, Mp = feats.shape[0], feats.shape[1]
    gen = torch.Generator(device='cpu').manual_seed(seed)
    history = []
    for ep in range(epochs):
        order = torch.randperm(P, generator=gen)
        tot = torch.zeros((), dtype=torch.float64, device='cuda')
        nb = 0
        for s in range(0, P - batch_pairs + 1, batch_pairs):
            idx = order[s:s + batch_pairs].cuda()
            F = feats[idx].reshape(-1, IN_DIM)
            T = labels[idx].reshape(-1, N_OUT)
            # padding rows (zero features, zero label) stay in the batch: they only ask f(0) = 0
            loss, grads = model.gradients(F, T, F.shape[0], weight=1.0 / (batch_pairs * Mp))
            model.adam(grads, lr=lr)
            tot += loss
            nb += 1
        history.append(float(tot) / max(nb, 1))
        if log:
            log(f'epoch {ep}: loss {history[-1]:.6f}')
    return history


def warm_start(matching, model, scales=(1.0,)):
    """Set matching.control['a0'] to the network's proposal when it lowers the objective, else keep zero momentum
    (the plain optimiser is the fallback). With several `scales`, the proposal is tried at each multiple and the
    best one is kept (one forward shot per scale). Returns (used_proposal, objective_at_proposal, objective_at_zero,
    chosen_scale)."""
    X0 = matching.x0
    faces_t = matching.data.faces
    a_prop = model.predict(X0, faces_t, matching.data.x1, matching.options['KparDiff'])
    zero = torch.zeros_like(a_prop)
    matching.obj = None
    obj_zero = matching.objectiveFun() if torch.equal(matching.control['a0'], zero) else None
    if obj_zero is None:
        matching.control['a0'] = zero
        matching.obj = None
        obj_zero = matching.objectiveFun()
    best, best_scale = obj_zero, None
    obj_prop = None
    for s in scales:
        # control - s * (-a_prop) = s * a_prop; updateTry keeps the trial only when it beats `best`
        o = matching.updateTry({'a0': -a_prop}, float(s), best)
        if obj_prop is None or (np.isfinite(o) and o < obj_prop):
            obj_prop = o
        if np.isfinite(o) and o < best:
            best, best_scale = o, float(s)
    used = best_scale is not None
    if used:
        matching.acceptVarTry()
    return used, obj_prop, obj_zero, best_scale


# ---------------------------------------------------------------------------------------------------------------
# Coarse-to-fine warm start
# ---------------------------------------------------------------------------------------------------------------
def mean_edge_length(vertices, faces):
    """Mean edge length of a triangulation (each interior edge counted twice, which does not change the mean of a
    closed mesh)."""
    v = np.asarray(vertices, dtype=np.float64)
    f = np.asarray(faces, dtype=np.int64)
    e = np.concatenate([v[f[:, 1]] - v[f[:, 0]], v[f[:, 2]] - v[f[:, 1]], v[f[:, 0]] - v[f[:, 2]]])
    return float(np.linalg.norm(e, axis=1).mean())


def prolong_momentum(x_coarse, a_coarse, x_fine, Kdef, width):
    """Momentum `a_coarse` on a coarse sampling of the source surface -> momentum on a finer sampling of the same
    surface with the same velocity field to first order. The momentum density m = a * mass (mass_k = sum_l
    K(x_k, x_l) under the deformation kernel Kdef; m has velocity units and does not depend on the sampling) is
    interpolated at the fine points by a normalised Gaussian of `width` (a fraction of the coarse edge length keeps
    it from smoothing the coarse solution) and divided by the fine kernel mass."""
    Xc, Xf = nat.as_device(x_coarse), nat.as_device(x_fine)
    m = nat.as_device(a_coarse) * kernel_mass(Kdef, Xc)
    Kh = Kernel(name='gauss', sigma=float(width))
    Kh.pk_dtype = 'float32'
    num = Kh.applyK(Xc, torch.cat([m, torch.ones_like(m[:, :1])], dim=1), firstVar=Xf)
    return (num[:, :3] / num[:, 3:4] / kernel_mass(Kdef, Xf)).contiguous()


class _CoarseConverged(Exception):
    pass


def _refine(matching, rtol, window):
    """The plain optimiser on `matching` until its objective decreases by less than `rtol` (relative) over `window`
    iterations, or its own stopping rule, or options['maxIter']."""
    end = matching.endOfIteration

    def end_of_iteration(endP=False):
        end(endP)
        h = matching.history
        if not endP and len(h) > window and (h[-1 - window] - h[-1]) <= rtol * abs(h[-1]):
            raise _CoarseConverged()

    matching.endOfIteration = end_of_iteration
    try:
        matching.optimizeMatching()
    except _CoarseConverged:
        pass
    finally:
        matching.endOfIteration = end


def multilevel_warm_start(matching, model, coarse_templates, rtol=1e-4, window=3, max_iter=200, width_factor=0.4,
                          scales=(0.5, 0.75, 1.0), first_step_gap=1e-3):
    """The learned warm start refined coarse to fine, for a SecondOrderSurfaceMatching `matching` (not yet
    optimised).

    `coarse_templates`: coarser triangulations (faces, vertices) of the same source surface, coarsest first. At the
    coarsest level the network (`model`; None for none) proposes a0 and `warm_start` keeps it when it lowers that
    level's objective; at every coarse level the plain optimiser (the same BFGS and objective, against the
    full-resolution target) refines the momentum until the objective decreases by less than `rtol` over `window`
    iterations (or `max_iter`), and `prolong_momentum` carries it to the next level (interpolation width
    `width_factor` x the coarse mean edge length). At the level of `matching` the prolonged momentum is the
    proposal: it becomes the control when it lowers the objective (the plain optimiser's zero start is the fallback),
    and `matching.optimizeMatching()` then refines from there, its first step along the gradient sized for a
    decrease of `first_step_gap` x the objective (`initial_step` of the matching; None: the optimiser's unit step,
    which at this distance from the optimum overshoots ~10^4-fold and costs ~5 extra objective evaluations).

    Returns a record: per level its vertex count, iterations and objective, whether the network's proposal was
    taken, and whether the fine level took the prolonged momentum."""
    from .surfaceMatching import SecondOrderSurfaceMatching
    from copy import deepcopy
    o = matching.options
    target = (matching.fv1.faces, matching.fv1.vertices)
    rec = {'levels': [], 'network_proposal_used': None}
    a_prev, x_prev, h_prev = None, None, None
    for faces, verts in coarse_templates:
        opts = dict(o)
        opts.update(KparDiff=deepcopy(o['KparDiff']), KparDist=deepcopy(o['KparDist']), maxIter=max_iter,
                    targetObjective=None, verb=False, processGroup=None, warmStart=None,
                    initialMomentum=None if a_prev is None else prolong_momentum(x_prev, a_prev, verts,
                                                                                  o['KparDiff'], h_prev))
        level = SecondOrderSurfaceMatching(Template=(faces, verts), Target=target, options=opts)
        if a_prev is None and model is not None:
            rec['network_proposal_used'] = warm_start(level, model, scales=scales)[0]
        _refine(level, rtol, window)
        a_prev, x_prev = level.control['a0'], np.asarray(verts, dtype=np.float64)
        h_prev = width_factor * mean_edge_length(verts, faces)
        rec['levels'].append({'vertices': int(x_prev.shape[0]), 'iters': len(level.history),
                              'objective': float(level.obj) if level.obj is not None else None})
        del level
    if a_prev is None:
        rec['prolonged_used'] = False
        return rec
    a_fine = prolong_momentum(x_prev, a_prev, matching.x0, o['KparDiff'], h_prev)
    matching.obj = None
    obj_here = matching.objectiveFun()
    o_try = matching.updateTry({'a0': matching.control['a0'] - a_fine}, 1.0, obj_here)
    used = bool(np.isfinite(o_try) and o_try < obj_here)
    if used:
        matching.acceptVarTry()
        matching.first_step_gap = first_step_gap
    rec.update(prolonged_used=used, obj_prolonged=float(o_try), obj_start=float(obj_here),
               first_step_gap=first_step_gap if used else None)
    return rec
