"""Float64 CPU restatement of the surface data terms (varifold, current, measure) and their vertex gradients.

Reference: base/surfaceDistances.py (varifold :280-573, current :22-140, measure :207-278) and the face
geometry of base/surfaces.py:326-351. The varifold gradient follows the pair formulation of
`varifoldNormGradient_pykeops` (:470-573), which needs O(F) memory, instead of the dense numpy variant.

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py).
"""
import numpy as np
from numba import njit, prange

from .kernels import apply_k, apply_diff_kt


def face_geometry(vertices, faces, weights=None):
    """centers, surfel = cross(v2-v1, v3-v1)/2, face_weights = mean of vertex weights (base/surfaces.py:326-351)."""
    v1, v2, v3 = vertices[faces[:, 0]], vertices[faces[:, 1]], vertices[faces[:, 2]]
    centers = (v1 + v2 + v3) / 3.0
    surfel = np.cross(v2 - v1, v3 - v1) / 2.0
    if weights is None:
        fw = np.ones(faces.shape[0])
    else:
        w = np.asarray(weights, dtype=np.float64)
        fw = (w[faces[:, 0]] + w[faces[:, 1]] + w[faces[:, 2]]) / 3.0
    return centers, surfel, fw


def _varifold_faces(vertices, faces, weights):
    c, s, fw = face_geometry(vertices, faces, weights)
    a = np.sqrt((s ** 2).sum(axis=1) + 1e-10)
    n = s / a[:, None]
    return c, n, a, a * fw, fw


@njit(parallel=True, cache=True)
def _varifold_pair_sum(c1, n1, w1, c2, n2, w2, inv2s2):
    out = np.zeros(c1.shape[0])
    for k in prange(c1.shape[0]):
        acc = 0.0
        for l in range(c2.shape[0]):
            r2 = (c1[k, 0] - c2[l, 0]) ** 2 + (c1[k, 1] - c2[l, 1]) ** 2 + (c1[k, 2] - c2[l, 2]) ** 2
            g = n1[k, 0] * n2[l, 0] + n1[k, 1] * n2[l, 1] + n1[k, 2] * n2[l, 2]
            acc += np.exp(-r2 * inv2s2) * w2[l] * (1.0 + g * g)
        out[k] = acc * w1[k]
    return out


def varifold_norm0(x1, faces1, sigma, weights1=None):
    """sum_kl K(c_k, c_l) a_k a_l (1 + (n_k.n_l)^2) over the target (base/surfaceDistances.py:292-302)."""
    c, n, _, aw, _ = _varifold_faces(x1, faces1, weights1)
    return float(_varifold_pair_sum(c, n, aw, c, n, aw, 0.5 / sigma ** 2).sum())


def varifold_norm_def(xdef, faces, x1, faces1, sigma, weights=None, weights1=None):
    """|fvDef|^2 - 2 <fvDef, fv1> in the unoriented varifold metric (base/surfaceDistances.py:335-353)."""
    c1, n1, _, aw1, _ = _varifold_faces(xdef, faces, weights)
    c2, n2, _, aw2, _ = _varifold_faces(x1, faces1, weights1)
    i2 = 0.5 / sigma ** 2
    return float(_varifold_pair_sum(c1, n1, aw1, c1, n1, aw1, i2).sum()
                 - 2.0 * _varifold_pair_sum(c1, n1, aw1, c2, n2, aw2, i2).sum())


@njit(parallel=True, cache=True)
def _varifold_grad_pairs(c1, n1, c2, n2, w2, inv2s2):
    """Per target face k: Z_k = sum_l e_kl w2_l [2g(n2_l - g n1_k) + (1+g^2) n1_k],
    D_k = sum_l e_kl w2_l (1+g^2) (c1_k - c2_l), S_k = sum_l e_kl w2_l (1+g^2)."""
    F = c1.shape[0]
    Z = np.zeros((F, 3))
    D = np.zeros((F, 3))
    S = np.zeros(F)
    for k in prange(F):
        z0 = z1 = z2 = 0.0
        d0 = d1 = d2 = 0.0
        s = 0.0
        for l in range(c2.shape[0]):
            e0, e1, e2 = c1[k, 0] - c2[l, 0], c1[k, 1] - c2[l, 1], c1[k, 2] - c2[l, 2]
            e = np.exp(-(e0 * e0 + e1 * e1 + e2 * e2) * inv2s2) * w2[l]
            g = n1[k, 0] * n2[l, 0] + n1[k, 1] * n2[l, 1] + n1[k, 2] * n2[l, 2]
            f = 1.0 + g * g
            z0 += e * (2.0 * g * (n2[l, 0] - g * n1[k, 0]) + f * n1[k, 0])
            z1 += e * (2.0 * g * (n2[l, 1] - g * n1[k, 1]) + f * n1[k, 1])
            z2 += e * (2.0 * g * (n2[l, 2] - g * n1[k, 2]) + f * n1[k, 2])
            d0 += e * f * e0
            d1 += e * f * e1
            d2 += e * f * e2
            s += e * f
        Z[k, 0], Z[k, 1], Z[k, 2] = z0, z1, z2
        D[k, 0], D[k, 1], D[k, 2] = d0, d1, d2
        S[k] = s
    return Z, D, S


def scatter_to_vertices(xdef, faces, dz1, z1):
    """px[v] += dz1_f - cross(opposite edge, z1_f) for each corner (base/surfaceDistances.py:435-453)."""
    x1, x2, x3 = xdef[faces[:, 0]], xdef[faces[:, 1]], xdef[faces[:, 2]]
    px = np.zeros_like(xdef)
    np.add.at(px, faces[:, 0], dz1 - np.cross(x3 - x2, z1))
    np.add.at(px, faces[:, 1], dz1 - np.cross(x1 - x3, z1))
    np.add.at(px, faces[:, 2], dz1 - np.cross(x2 - x1, z1))
    return px


def varifold_norm_gradient(xdef, faces, x1, faces1, sigma, weights=None, weights1=None, with_weights=False):
    """Gradient of varifoldNormDef with respect to the deformed vertices (base/surfaceDistances.py:470-573)."""
    c1, n1, a1, aw1, fw1 = _varifold_faces(xdef, faces, weights)
    c2, n2, _, aw2, _ = _varifold_faces(x1, faces1, weights1)
    i2 = 0.5 / sigma ** 2
    Za, Da, Sa = _varifold_grad_pairs(c1, n1, c1, n1, aw1, i2)
    Zb, Db, Sb = _varifold_grad_pairs(c1, n1, c2, n2, aw2, i2)
    z1 = fw1[:, None] * (Za - Zb)
    dz1 = -(2.0 / 3.0) * (aw1 / sigma ** 2)[:, None] * (Da - Db)
    px = scatter_to_vertices(xdef, faces, dz1, z1)
    if not with_weights:
        return px
    z1w = (2.0 / 3.0) * fw1 * a1 * (Sa - Sb)
    pxw = np.zeros(xdef.shape[0])
    for j in range(3):
        np.add.at(pxw, faces[:, j], z1w)
    return px, pxw


def varifold_norm_gradient_rows(xdef, faces, x1, faces1, sigma, vertices):
    """varifold_norm_gradient at the listed vertices only (unit weights): the pair sums run for the faces incident to
    those vertices, whose per-face terms are all that the scatter of base/surfaceDistances.py:435-453 adds to them."""
    vertices = np.asarray(vertices, dtype=np.int64)
    mark = np.zeros(xdef.shape[0], dtype=bool)
    mark[vertices] = True
    sel = np.nonzero(mark[faces].any(axis=1))[0]
    c1, n1, _, aw1, fw1 = _varifold_faces(xdef, faces, None)
    c2, n2, _, aw2, _ = _varifold_faces(x1, faces1, None)
    i2 = 0.5 / sigma ** 2
    cs, ns = np.ascontiguousarray(c1[sel]), np.ascontiguousarray(n1[sel])
    Za, Da, _ = _varifold_grad_pairs(cs, ns, c1, n1, aw1, i2)
    Zb, Db, _ = _varifold_grad_pairs(cs, ns, c2, n2, aw2, i2)
    z1 = np.zeros((faces.shape[0], 3))
    dz1 = np.zeros((faces.shape[0], 3))
    z1[sel] = fw1[sel, None] * (Za - Zb)
    dz1[sel] = -(2.0 / 3.0) * (aw1[sel] / sigma ** 2)[:, None] * (Da - Db)
    return scatter_to_vertices(xdef, faces, dz1, z1)[vertices]


def current_norm0(x1, faces1, sigma, weights1=None):
    """sum_k cr_k . (K cr)_k with cr = face_weights * surfel (base/surfaceDistances.py:22-26, :70)."""
    c, s, fw = face_geometry(x1, faces1, weights1)
    cr = s * fw[:, None]
    return float((cr * apply_k(c, c, cr, sigma)).sum())


def current_norm_def(xdef, faces, x1, faces1, sigma, weights=None, weights1=None):
    """(base/surfaceDistances.py:75-81)."""
    c1, s1, f1 = face_geometry(xdef, faces, weights)
    c2, s2, f2 = face_geometry(x1, faces1, weights1)
    cr1, cr2 = s1 * f1[:, None], s2 * f2[:, None]
    return float((cr1 * apply_k(c1, c1, cr1, sigma)).sum() - 2.0 * (cr1 * apply_k(c1, c2, cr2, sigma)).sum())


def current_norm_gradient(xdef, faces, x1, faces1, sigma, weights=None, weights1=None):
    """(base/surfaceDistances.py:90-133)."""
    c1, s1, f1 = face_geometry(xdef, faces, weights)
    c2, s2, f2 = face_geometry(x1, faces1, weights1)
    w1, w2 = s1 * f1[:, None], s2 * f2[:, None]
    z1 = apply_k(c1, c1, w1, sigma) - apply_k(c1, c2, w2, sigma)
    wz1 = f1[:, None] * z1
    dz1 = (2.0 / 3.0) * (apply_diff_kt(c1, c1, w1, w1, sigma) - apply_diff_kt(c1, c2, w1, w2, sigma))
    return scatter_to_vertices(xdef, faces, dz1, wz1)


def _measure_faces(vertices, faces, weights):
    c, s, fw = face_geometry(vertices, faces, weights)
    a = np.sqrt((s ** 2).sum(axis=1) + 1e-10)
    return c, s / a[:, None], a, a * fw, fw


def measure_norm0(x1, faces1, sigma, weights1=None):
    """(base/surfaceDistances.py:207-211)."""
    c, _, _, aw, _ = _measure_faces(x1, faces1, weights1)
    return float((aw * apply_k(c, c, aw[:, None], sigma)[:, 0]).sum())


def measure_norm_def(xdef, faces, x1, faces1, sigma, weights=None, weights1=None):
    """(base/surfaceDistances.py:215-223)."""
    c1, _, _, aw1, _ = _measure_faces(xdef, faces, weights)
    c2, _, _, aw2, _ = _measure_faces(x1, faces1, weights1)
    return float((aw1 * apply_k(c1, c1, aw1[:, None], sigma)[:, 0]).sum()
                 - 2.0 * (aw1 * apply_k(c1, c2, aw2[:, None], sigma)[:, 0]).sum())


@njit(parallel=True, cache=True)
def _scalar_diff_kt(y, x, p, a, inv2s2):
    out = np.zeros((y.shape[0], 3))
    for k in prange(y.shape[0]):
        for l in range(x.shape[0]):
            d0, d1, d2 = y[k, 0] - x[l, 0], y[k, 1] - x[l, 1], y[k, 2] - x[l, 2]
            f = np.exp(-(d0 * d0 + d1 * d1 + d2 * d2) * inv2s2) * p[k] * a[l] * (-2.0 * inv2s2)
            out[k, 0] += f * d0
            out[k, 1] += f * d1
            out[k, 2] += f * d2
    return out


def measure_norm_gradient(xdef, faces, x1, faces1, sigma, weights=None, weights1=None):
    """(base/surfaceDistances.py:232-278)."""
    c1, n1, _, aw1, f1 = _measure_faces(xdef, faces, weights)
    c2, _, _, aw2, _ = _measure_faces(x1, faces1, weights1)
    z1 = apply_k(c1, c1, aw1[:, None], sigma)[:, 0] - apply_k(c1, c2, aw2[:, None], sigma)[:, 0]
    wz1 = (f1 * z1)[:, None] * n1
    i2 = 0.5 / sigma ** 2
    dz1 = (2.0 / 3.0) * (_scalar_diff_kt(c1, c1, aw1, aw1, i2) - _scalar_diff_kt(c1, c2, aw1, aw2, i2))
    return scatter_to_vertices(xdef, faces, dz1, wz1)
