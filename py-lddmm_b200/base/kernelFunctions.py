"""Drop-in `Kernel` / `KernelSpec` (reference: base/kernelFunctions.py:337-680) backed by the sm_100a library.

Signatures, argument meaning and return shapes follow the reference. Inputs may be numpy arrays (the
reference's contract: numpy in, new numpy array out, inputs never written) or torch tensors (CUDA or CPU);
the result has the type of `x`. Every sum runs in the CUDA library (no CPU fallback).

Supported: the Gaussian kernel ('gauss' / 'gaussian') and the reference's Laplacian (Matern) kernel
('laplacian', order 0..4: P_order(r/sigma) exp(-r/sigma), base/kernelFunctions_util.py:20-56), with one or several
widths (multi-scale sums weighted by sigma**ms_exponent / sum(sigma**ms_exponent),
base/kernelFunctions_util.py:451-466), affine='none'. applyKTensor and the dense-weight variants (matrixWeights,
applyDiffKmat) are Gaussian only, as are the surface data terms.
`pk_dtype` selects the arithmetic: 'float32' -> FP32 pair sums with compensated accumulation,
'float64' -> FP64 pair sums (the faithful path); both return float64 like the reference.
"""
import logging

import numpy as np
import torch

from . import _native as nat

_GAUSS = ('gauss', 'gaussian')
_FAMILIES = _GAUSS + ('laplacian',)
# lapPol coefficients of the Laplacian kernel by order (base/kernelFunctions_util.py:20-24)
_LAP_POLY = ((1, 0, 0, 0, 0), (1, 1, 0, 0, 0), (1, 1, 1 / 3, 0, 0), (1, 1, 0.4, 1 / 15, 0),
             (1, 1, 3 / 7, 2 / 21, 1 / 105))


def _is_np(v):
    return not isinstance(v, torch.Tensor)


_NO_ORIGIN = object()   # marks calls whose kernel needs no coordinate origin


def _out(t, like_numpy):
    return nat.to_host(t) if like_numpy else t


class KernelSpec:
    """Kernel parameters (base/kernelFunctions.py:337-412)."""

    def __init__(self, name='gauss', affine='none', sigma=(1.,), order=3, w1=1.0, w2=1.0, dim=3, weight=1.0,
                 localMaps=None):
        self.name = name
        self.sigma = np.array([sigma], dtype=float) if np.isscalar(sigma) else np.array(sigma, dtype=float)
        self.order = order
        self.weight = weight
        self.dim = dim
        self.affine_basis = []
        self.precomp = []
        self._hold = False
        self._state = False
        self.localMaps = localMaps
        self.setAffine(affine, w1, w2)
        self.kff = name in _FAMILIES
        self.pk_dtype = 'float64'
        self.ms_exponent = -1
        if name == 'laplacian':
            if self.order > 4:
                self.order = 3
            self.par = [sigma, self.order]
        elif name in _GAUSS:
            self.order = 10
            self.par = [sigma]
        else:
            self.par = []

    def setAffine(self, affine, w1=1., w2=1., center=None):
        self.affine = affine
        self.w1 = w1
        self.w2 = w2
        self.center = np.zeros(self.dim) if center is None else np.array(center)


class Kernel(KernelSpec):
    """Gaussian kernel operators on the B200 (base/kernelFunctions.py:414-680)."""

    # ------------------------------------------------------------------ helpers
    def _check(self, gauss_only=False):
        if self.name not in (_GAUSS if gauss_only else _FAMILIES):
            what = 'the Gaussian kernel' if gauss_only else "the 'gauss' and 'laplacian' kernels"
            raise NotImplementedError(f"lddmm_b200 implements {what} here (got '{self.name}')")
        if self.affine not in (None, 'none'):
            raise NotImplementedError("lddmm_b200 implements affine='none' only")
        if self.localMaps:
            raise NotImplementedError('lddmm_b200 does not implement localMaps kernels')

    @property
    def code(self):
        """Kernel-family argument of the library (0: Gaussian, 16 + order: Laplacian)."""
        return nat.kernel_code(self)

    @property
    def precision(self):
        return nat.FP64 if str(self.pk_dtype) in ('float64', 'double') else nat.FP32C

    def _scales(self):
        s = np.asarray(self.sigma, dtype=float).ravel()
        w = s ** self.ms_exponent
        return list(zip(s.tolist(), (w / w.sum()).tolist()))

    def _multi(self, fn):
        """sum_s w_s fn(sigma_s); one launch per width."""
        scales = self._scales()
        if len(scales) == 1 and scales[0][1] == 1.0:
            return fn(scales[0][0])        # one width: no weighting pass
        res = None
        for s, w in scales:
            r = fn(s)
            res = r * w if res is None else res + r * w
        return res

    # ------------------------------------------------------------------ K
    def applyK(self, x, a, firstVar=None, grid=None, matrixWeights=False, cpu=False):
        """K(x,x)a or K(firstVar, x)a (base/kernelFunctions.py:452-506); matrixWeights -> sum_l K_kl a[k,l,:]."""
        self._check()
        like_np = _is_np(x)
        X = nat.as_device(x)
        Y = X if firstVar is None else nat.as_device(firstVar)
        if matrixWeights:
            self._check(gauss_only=True)
            U = nat.as_device(a)
            if U.dim() == 2:
                U = U[..., None]
            r = self._multi(lambda s: self._k_mat(Y, X, U, s))
            return _out(r, like_np)
        A = nat.as_device(a)
        squeeze = A.dim() == 1
        if squeeze:
            A = A[:, None]
        # The Gaussian sums run the expanded-distance kernel (FP32) or FP64 arithmetic, both of which take coordinates
        # relative to each target block's own centre in FP64: no origin is needed, and the host pass that computes one
        # is skipped. The Laplacian FP32 kernel evaluates differences of origin-centred FP32 coordinates.
        origin = _NO_ORIGIN if self.code == nat.KERNEL_GAUSS else nat.centroid(x)
        if A.shape[1] != 3:
            r = self._multi(lambda s: self._k_generic(Y, X, A, s, origin))
        else:
            r = self._multi(lambda s: self._apply_k(Y, X, A, s, origin))
        if squeeze:
            r = r[:, 0]
        return _out(r, like_np)

    def _apply_k(self, Y, X, A, sigma, origin=None):
        n, m = Y.shape[0], X.shape[0]
        out = torch.empty((n, 3), dtype=torch.float64, device=Y.device)
        ws, wsb = nat.workspace(n, m, self.precision)
        o = None if origin is _NO_ORIGIN else nat.origin_arg(origin if origin is not None else nat.centroid(X))
        nat.check(nat.lib().lddmm_apply_k(nat.ptr(Y), n, nat.ptr(X), nat.ptr(A), m, float(sigma), self.code, o,
                                          nat.ptr(out), self.precision, ws, wsb, nat.stream_ptr()), 'applyK')
        return out

    def _k_generic(self, Y, X, A, sigma, origin=None):
        """K a for momenta of any width d: columns in groups of 3 (zero padded)."""
        d = A.shape[1]
        cols = []
        for c0 in range(0, d, 3):
            blk = A[:, c0:c0 + 3]
            if blk.shape[1] < 3:
                blk = torch.cat([blk, blk.new_zeros(blk.shape[0], 3 - blk.shape[1])], dim=1)
            cols.append(self._apply_k(Y, X, blk.contiguous(), sigma, origin))
        return torch.cat(cols, dim=1)[:, :d].contiguous()

    def _k_mat(self, Y, X, U, sigma):
        n, m, d = Y.shape[0], X.shape[0], U.shape[2]
        out = torch.empty((n, d), dtype=torch.float64, device=Y.device)
        nat.check(nat.lib().lddmm_apply_k_mat(nat.ptr(Y), n, nat.ptr(X), m, nat.ptr(U.contiguous()), d, float(sigma),
                                              nat.ptr(out), nat.stream_ptr()), 'applyK(matrixWeights)')
        return out

    def applyKTensor(self, x, ay, ax, betay, betax, firstVar=None, grid=None, cpu=False):
        """sum_l K_kl (ay_k ax_l + (betay_k.betax_l)^2) (base/kernelFunctions.py:509-517)."""
        self._check(gauss_only=True)
        like_np = _is_np(x)
        X = nat.as_device(x)
        Y = X if firstVar is None else nat.as_device(firstVar)
        AY, AX = nat.as_device(ay).reshape(-1), nat.as_device(ax).reshape(-1)
        BY, BX = nat.as_device(betay), nat.as_device(betax)
        n, m = Y.shape[0], X.shape[0]
        o = nat.origin_arg(nat.centroid(X))

        def one(s):
            out = torch.empty(n, dtype=torch.float64, device=Y.device)
            ws, wsb = nat.workspace(n, m, self.precision)
            nat.check(nat.lib().lddmm_apply_k_tensor(nat.ptr(Y), n, nat.ptr(X), m, nat.ptr(AY), nat.ptr(AX),
                                                     nat.ptr(BY), nat.ptr(BX), float(s), o, nat.ptr(out),
                                                     self.precision, ws, wsb, nat.stream_ptr()), 'applyKTensor')
            return out
        return _out(self._multi(one), like_np)

    # ------------------------------------------------------------------ first derivatives
    def _diff_k1and2(self, X, A1, A2, sigma):
        """-(1/sigma^2) sum_l (D.(A1_k - A1_l)) K_kl A2_l for one width."""
        n = X.shape[0]
        out = torch.empty((n, 3), dtype=torch.float64, device=X.device)
        ws, wsb = nat.workspace(n, n, self.precision)
        o = nat.origin_arg(nat.centroid(X))
        nat.check(nat.lib().lddmm_apply_diff_k1and2(nat.ptr(X), nat.ptr(A1), nat.ptr(A2), n, float(sigma), self.code,
                                                    o, nat.ptr(out), self.precision, ws, wsb, nat.stream_ptr()),
                  'applyDiffK1and2')
        return out

    def applyDiffK1and2(self, x, a1, a2):
        """A_k = sum_l D_1[K(x_k,x_l) a2_l](a1_k) + D_2[...](a1_l) (base/kernelFunctions.py:549-562)."""
        self._check()
        like_np = _is_np(x)
        X, A1, A2 = nat.as_device(x), nat.as_device(a1), nat.as_device(a2)
        return _out(self._multi(lambda s: self._diff_k1and2(X, A1, A2, s)), like_np)

    def _diff_k2(self, X, A1, A2):
        """opt2_k = (1/s^2) sum_l (D.a1_l) K_kl a2_l (ku option '2'), evaluated as DK1and2 on the stacked set
        [X; X] with a1 = [0; a1], a2 = [0; a2]: for a target of the first half, D.(0 - a1_l) = -(D.a1_l) and only
        the second half contributes."""
        n = X.shape[0]
        XX = torch.cat([X, X], dim=0)
        A1s = torch.cat([torch.zeros_like(A1), A1], dim=0)
        A2s = torch.cat([torch.zeros_like(A2), A2], dim=0)
        return self._multi(lambda s: self._diff_k1and2(XX, A1s, A2s, s))[:n]

    def applyDiffK(self, x, a1, a2):
        """A_k = sum_l D_1[K(x_k, x_l) a2_l] a1_k (base/kernelFunctions.py:520-532) = DK1and2 - opt2."""
        self._check()
        like_np = _is_np(x)
        X, A1, A2 = nat.as_device(x), nat.as_device(a1), nat.as_device(a2)
        r = self._multi(lambda s: self._diff_k1and2(X, A1, A2, s)) - self._diff_k2(X, A1, A2)
        return _out(r, like_np)

    def applyDiffK2(self, x, a1, a2):
        """A_k = sum_l D_2[K(x_k, x_l) a2_l] a1_l (base/kernelFunctions.py:535-546): +(1/s^2) sum (D.a1_l) K a2_l."""
        self._check()
        like_np = _is_np(x)
        X, A1, A2 = nat.as_device(x), nat.as_device(a1), nat.as_device(a2)
        return _out(self._diff_k2(X, A1, A2), like_np)

    def applyDiffKmat(self, x, beta, firstVar=None):
        """sum_l -(y_k - x_l)/sigma^2 K_kl beta[k,l] (base/kernelFunctions.py:565-570)."""
        self._check(gauss_only=True)
        like_np = _is_np(x)
        X = nat.as_device(x)
        Y = X if firstVar is None else nat.as_device(firstVar)
        B = nat.as_device(beta)
        n, m = Y.shape[0], X.shape[0]

        def one(s):
            out = torch.empty((n, 3), dtype=torch.float64, device=Y.device)
            nat.check(nat.lib().lddmm_apply_diff_k_mat(nat.ptr(Y), n, nat.ptr(X), m, nat.ptr(B), float(s),
                                                       nat.ptr(out), nat.stream_ptr()), 'applyDiffKmat')
            return out
        return _out(self._multi(one), like_np)

    def applyDiffKT(self, x, p0, a, firstVar=None, regweight=1., lddmm=False, sym=False, extra_term=None, cpu=False):
        """sum_l -(y_k - x_l)/sigma^2 K_kl c_kl (base/kernelFunctions.py:581-626)."""
        self._check()
        like_np = _is_np(x)
        X = nat.as_device(x)
        Y = X if firstVar is None else nat.as_device(firstVar)
        P, A = nat.as_device(p0), nat.as_device(a)
        if P.dim() == 3:   # (1, N, 3) forms used by some reference callers
            P = P.reshape(-1, 3)
        if A.dim() == 3:
            A = A.reshape(-1, 3)
        if lddmm and extra_term is not None:
            P = P + nat.as_device(extra_term)
        mode = 2 if lddmm else (1 if sym else 0)
        n, m = Y.shape[0], X.shape[0]
        if A.shape[1] != 3 or P.shape[1] != 3:
            if mode != 0:
                raise NotImplementedError('sym/lddmm applyDiffKT needs 3-vectors')
            # c_kl = p_k . a_l for d-vectors: sum over groups of 3 coordinates
            d = A.shape[1]
            pad = (-d) % 3
            if pad:
                A = torch.cat([A, A.new_zeros(A.shape[0], pad)], 1)
                P = torch.cat([P, P.new_zeros(P.shape[0], pad)], 1)
            r = None
            for c0 in range(0, d + pad, 3):
                rr = self._diff_kt(Y, X, P[:, c0:c0 + 3].contiguous(), A[:, c0:c0 + 3].contiguous(), 0, regweight)
                r = rr if r is None else r + rr
            return _out(r, like_np)
        return _out(self._diff_kt(Y, X, P, A, mode, regweight), like_np)

    def _diff_kt(self, Y, X, P, A, mode, regweight, origin=None):
        n, m = Y.shape[0], X.shape[0]
        o = nat.origin_arg(origin if origin is not None else nat.centroid(X))

        def one(s):
            out = torch.empty((n, 3), dtype=torch.float64, device=Y.device)
            ws, wsb = nat.workspace(n, m, self.precision)
            nat.check(nat.lib().lddmm_apply_diff_kt(nat.ptr(Y), n, nat.ptr(X), nat.ptr(P), nat.ptr(A), m, float(s),
                                                    self.code, mode, float(regweight), o, nat.ptr(out),
                                                    self.precision, ws, wsb, nat.stream_ptr()), 'applyDiffKT')
            return out
        return self._multi(one)

    def testDiffKT(self, y, x, p, a):
        """Finite-difference probe of applyDiffKT (base/kernelFunctions.py:629-635); returns (fd, analytic)."""
        k0 = (p * self.applyK(x, a, firstVar=y)).sum()
        dy = np.random.randn(y.shape[0], y.shape[1])
        eps = 1e-8
        k1 = (p * self.applyK(x, a, firstVar=y + eps * dy)).sum()
        grd = self.applyDiffKT(x, p, a, firstVar=y)
        fd, an = float((k1 - k0) / eps), float((grd * dy).sum())
        logging.info(f'applyDiffKT check: finite difference {fd:.5f}, analytic {an:.5f}')
        return fd, an

    def applyDivergence(self, x, a, firstVar=None):
        """sum_l -((y_k - x_l).a_l)/sigma^2 K_kl, shape (N,1) (base/kernelFunctions.py:638-662)."""
        self._check()
        like_np = _is_np(x)
        X = nat.as_device(x)
        Y = X if firstVar is None else nat.as_device(firstVar)
        A = nat.as_device(a)
        n, m = Y.shape[0], X.shape[0]
        o = nat.origin_arg(nat.centroid(X))

        def one(s):
            out = torch.empty((n, 1), dtype=torch.float64, device=Y.device)
            ws, wsb = nat.workspace(n, m, self.precision)
            nat.check(nat.lib().lddmm_apply_divergence(nat.ptr(Y), n, nat.ptr(X), nat.ptr(A), m, float(s), self.code,
                                                       o, nat.ptr(out), self.precision, ws, wsb, nat.stream_ptr()),
                      'applyDivergence')
            return out
        return _out(self._multi(one), like_np)

    # ------------------------------------------------------------------ second derivative
    def applyDDiffK11and12(self, x, n, a, p):
        """sum_l (n_k.a_l) [D_11 + D_12] K_kl p (base/kernelFunctions.py:665-674)."""
        self._check()
        like_np = _is_np(x)
        X, Nn, A, P = nat.as_device(x), nat.as_device(n), nat.as_device(a), nat.as_device(p)
        N = X.shape[0]
        o = nat.origin_arg(nat.centroid(X))

        def one(s):
            out = torch.empty((N, 3), dtype=torch.float64, device=X.device)
            ws, wsb = nat.workspace(N, N, self.precision)
            nat.check(nat.lib().lddmm_apply_ddiff_k11and12(nat.ptr(X), nat.ptr(Nn), nat.ptr(A), nat.ptr(P), N,
                                                           float(s), self.code, o, nat.ptr(out), self.precision, ws,
                                                           wsb, nat.stream_ptr()), 'applyDDiffK11and12')
            return out
        return _out(self._multi(one), like_np)

    # ------------------------------------------------------------------ dense matrix / solve
    def getK(self, x, firstVar=None):
        """Dense kernel matrix (ku.kernelmatrix), computed on the device in FP64."""
        self._check()
        like_np = _is_np(x)
        X = nat.as_device(x)
        Y = X if firstVar is None else nat.as_device(firstVar)
        d2 = ((Y[:, None, :] - X[None, :, :]) ** 2).sum(-1)
        if self.name == 'laplacian':
            c = _LAP_POLY[int(self.order)]
            r = torch.sqrt(d2)

            def lap(s):
                u = r / s
                return (c[0] + u * (c[1] + u * (c[2] + u * (c[3] + u * c[4])))) * torch.exp(-u)
            K = self._multi(lap)
        else:
            K = self._multi(lambda s: torch.exp(-d2 / (2 * s * s)))
        return _out(K, like_np)

    def hold(self):
        self._state = self._hold
        self._hold = True

    def release(self):
        self._state = False
        self._hold = False

    def reset(self):
        self._hold = self._state

    def solve(self, x, xi, b, iterMax=100):
        """Conjugate-gradient solve with the operator a -> K(x) a (base/kernelFunctions.py:676-680)."""
        from .conjugateGradient import linearcg
        return linearcg(lambda a_: self.applyK(x, a_), xi, iterMax=iterMax)
