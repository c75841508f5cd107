"""Drop-in surface data terms (reference: base/surfaceDistances.py:22-573) on the B200.

`SurfaceDataTerm` is the device-resident form used by the matching drivers: it keeps the target surface,
the faces and the vertex->face incidence table on the GPU and evaluates energy and vertex gradient of the
deformed surface with two / three kernel launches. The reference-signature functions (varifoldNorm0,
varifoldNormDef, varifoldNormGradient, currentNorm*, measureNorm*) wrap it; they accept the reference's
`Surface` objects and return floats / numpy arrays.

Only the default varifold weight f0(u) = 1 + u^2 (`fun=None`) is implemented.
"""
import hashlib

import numpy as np
import torch

from . import _native as nat

KINDS = {'varifold': nat.DATA_VARIFOLD, 'current': nat.DATA_CURRENT, 'measure': nat.DATA_MEASURE}

_TABLES = {}


def vertex_face_table(faces_np, nv):
    """(offsets (nv+1) int32, items (3F) int32) on the device, cached per topology."""
    faces_np = np.ascontiguousarray(faces_np, dtype=np.int64)
    key = (hashlib.sha1(faces_np.tobytes()).hexdigest(), int(nv), torch.cuda.current_device())
    hit = _TABLES.get(key)
    if hit is not None:
        return hit
    off = np.zeros(nv + 1, dtype=np.int32)
    items = np.zeros(max(3 * faces_np.shape[0], 1), dtype=np.int32)
    rc = nat.lib().lddmm_vertex_face_table(faces_np.ctypes.data, faces_np.shape[0], int(nv), off.ctypes.data,
                                           items.ctypes.data)
    nat.check(rc, 'vertex_face_table')
    val = (torch.from_numpy(off).cuda(), torch.from_numpy(items).cuda())
    if len(_TABLES) > 32:
        _TABLES.clear()
    _TABLES[key] = val
    return val


def _kernel_widths(KparDist):
    if isinstance(KparDist, (int, float)):
        return [(float(KparDist), 1.0)], nat.FP32C
    if KparDist.name not in ('gauss', 'gaussian'):
        raise NotImplementedError('lddmm_b200 data terms use the Gaussian kernel only')
    s = np.asarray(KparDist.sigma, dtype=float).ravel()
    w = s ** KparDist.ms_exponent
    prec = nat.FP64 if str(getattr(KparDist, 'pk_dtype', 'float64')) in ('float64', 'double') else nat.FP32C
    return list(zip(s.tolist(), (w / w.sum()).tolist())), prec


class SurfaceDataTerm:
    """Device-resident data term |S_def|^2 - 2<S_def, S_1> (+ |S_1|^2) for a fixed topology and target."""

    def __init__(self, faces, target_vertices, target_faces, KparDist, kind='varifold', weights=None,
                 target_weights=None, precision=None, nv=None):
        self.kind = KINDS[kind] if isinstance(kind, str) else int(kind)
        self.widths, prec = _kernel_widths(KparDist)
        self.precision = prec if precision is None else precision
        self.faces_np = np.ascontiguousarray(faces, dtype=np.int64)
        self.faces = torch.from_numpy(self.faces_np).cuda()
        self.nf = self.faces_np.shape[0]
        self.nv = int(nv) if nv is not None else int(self.faces_np.max()) + 1
        self.x1 = nat.as_device(target_vertices)
        f1 = np.ascontiguousarray(target_faces, dtype=np.int64)
        if f1.size and (f1.min() < 0 or f1.max() >= self.x1.shape[0]):
            raise ValueError('target faces index outside the target vertices')
        if f1.ndim != 2 or f1.shape[1] != 3 or self.faces_np.ndim != 2 or self.faces_np.shape[1] != 3:
            raise ValueError('faces must be (F, 3) triangles')
        self.faces1 = torch.from_numpy(f1).cuda()
        self.nf1 = self.faces1.shape[0]
        self.w = None if weights is None else nat.as_device(weights)
        self.w1 = None if target_weights is None else nat.as_device(target_weights)
        self.vf_off, self.vf_items = vertex_face_table(self.faces_np, self.nv)
        self.origin = nat.centroid(self.x1)
        self._norm0 = None

    def _ws(self):
        return nat.surface_workspace(self.nf, self.nf1, self.precision)

    def energy(self, xdef, with_norm0=False):
        """Device tensor (2,): [xNormDef, xNorm0 (or 0)] in FP64. xdef=None evaluates xNorm0 only."""
        X = None if xdef is None else nat.as_device(xdef)
        nv, nf = (0, 0) if X is None else (X.shape[0], self.nf)
        out = torch.zeros(2, dtype=torch.float64, device=self.x1.device)
        tmp = torch.empty(2, dtype=torch.float64, device=self.x1.device)
        ws, wsb = self._ws()
        o = nat.origin_arg(self.origin)
        for s, wt in self.widths:
            nat.check(nat.lib().lddmm_surface_energy(self.kind, nat.ptr(X), nv, nat.ptr(self.faces), nf,
                                                     nat.ptr(self.w), nat.ptr(self.x1), self.x1.shape[0],
                                                     nat.ptr(self.faces1), self.nf1, nat.ptr(self.w1), float(s), o,
                                                     int(bool(with_norm0)), nat.ptr(tmp), self.precision, ws, wsb,
                                                     nat.stream_ptr()), 'surface_energy')
            if not with_norm0:
                tmp[1] = 0.0
            out += wt * tmp
        return out

    def norm0(self):
        """|S_1|^2 (cached host float)."""
        if self._norm0 is None:
            self._norm0 = float(self.energy(None, with_norm0=True)[1])
        return self._norm0

    def gradient(self, xdef, with_weights=False):
        """Vertex gradient of xNormDef, (nv,3) FP64 device tensor (and (nv,) weight gradient if requested)."""
        X = nat.as_device(xdef)
        px = torch.zeros((X.shape[0], 3), dtype=torch.float64, device=X.device)
        pxw = torch.zeros(X.shape[0], dtype=torch.float64, device=X.device) if with_weights else None
        tmp = torch.empty_like(px)
        tmpw = torch.empty_like(pxw) if with_weights else None
        ws, wsb = self._ws()
        o = nat.origin_arg(self.origin)
        for s, wt in self.widths:
            nat.check(nat.lib().lddmm_surface_gradient(self.kind, nat.ptr(X), X.shape[0], nat.ptr(self.faces),
                                                       self.nf, nat.ptr(self.w), nat.ptr(self.vf_off),
                                                       nat.ptr(self.vf_items), nat.ptr(self.x1), self.x1.shape[0],
                                                       nat.ptr(self.faces1), self.nf1, nat.ptr(self.w1), float(s), o,
                                                       nat.ptr(tmp), nat.ptr(tmpw), self.precision, ws, wsb,
                                                       nat.stream_ptr()), 'surface_gradient')
            px += wt * tmp
            if with_weights:
                pxw += wt * tmpw
        return (px, pxw) if with_weights else px


def _weights(fv):
    w = getattr(fv, 'weights', None)
    if w is None:
        return None
    w = np.asarray(w, dtype=np.float64)
    return None if np.all(w == 1.0) else w


def _term(fvDef, fv1, KparDist, kind):
    return SurfaceDataTerm(fvDef.faces, fv1.vertices, fv1.faces, KparDist, kind=kind, weights=_weights(fvDef),
                           target_weights=_weights(fv1), nv=fvDef.vertices.shape[0])


def _self_term(fv1, KparDist, kind):
    return SurfaceDataTerm(fv1.faces, fv1.vertices, fv1.faces, KparDist, kind=kind, weights=_weights(fv1),
                           target_weights=_weights(fv1), nv=fv1.vertices.shape[0])


def _check_fun(fun):
    if fun is not None:
        raise NotImplementedError('lddmm_b200 implements the default varifold weight f0(u) = 1 + u^2 only')


# --- varifold (base/surfaceDistances.py:280-573) ---------------------------------------------------------------
def varifoldNorm0(fv1, KparDist, fun=None, cpu=False, dtype='float64'):
    _check_fun(fun)
    return _self_term(fv1, KparDist, 'varifold').norm0()


def varifoldNormDef(fvDef, fv1, KparDist, fun=None, cpu=False, dtype='float64'):
    _check_fun(fun)
    return float(_term(fvDef, fv1, KparDist, 'varifold').energy(fvDef.vertices)[0])


def varifoldNorm(fvDef, fv1, KparDist, fun=None):
    return varifoldNormDef(fvDef, fv1, KparDist, fun=fun) + varifoldNorm0(fv1, KparDist, fun=fun)


def varifoldNormGradient(fvDef, fv1, KparDist, with_weights=False, fun=None, cpu=False, dtype='float64'):
    _check_fun(fun)
    r = _term(fvDef, fv1, KparDist, 'varifold').gradient(fvDef.vertices, with_weights=with_weights)
    if with_weights:
        return r[0].cpu().numpy(), r[1].cpu().numpy()
    return r.cpu().numpy()


# --- current (base/surfaceDistances.py:22-133) -------------------------------------------------------------------
def currentNorm0(fv1, KparDist, weight=1.):
    return _self_term(fv1, KparDist, 'current').norm0()


def currentNormDef(fvDef, fv1, KparDist, weight=1.):
    return float(_term(fvDef, fv1, KparDist, 'current').energy(fvDef.vertices)[0])


def currentNorm(fvDef, fv1, KparDist, weight=1.):
    return currentNormDef(fvDef, fv1, KparDist) + currentNorm0(fv1, KparDist)


def currentNormGradient(fvDef, fv1, KparDist, weight=1., with_weights=False):
    if with_weights:
        raise NotImplementedError('with_weights is implemented for the varifold only')
    return _term(fvDef, fv1, KparDist, 'current').gradient(fvDef.vertices).cpu().numpy()


# --- measure (base/surfaceDistances.py:207-278) -------------------------------------------------------------------
def measureNorm0(fv1, KparDist):
    return _self_term(fv1, KparDist, 'measure').norm0()


def measureNormDef(fvDef, fv1, KparDist):
    return float(_term(fvDef, fv1, KparDist, 'measure').energy(fvDef.vertices)[0])


def measureNorm(fvDef, fv1, KparDist):
    return measureNormDef(fvDef, fv1, KparDist) + measureNorm0(fv1, KparDist)


def measureNormGradient(fvDef, fv1, KparDist, with_weights=False):
    if with_weights:
        raise NotImplementedError('with_weights is implemented for the varifold only')
    return _term(fvDef, fv1, KparDist, 'measure').gradient(fvDef.vertices).cpu().numpy()
