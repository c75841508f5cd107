"""Synthetic surfaces used by the benchmarks, the parity fixtures and the learned proposal.

The reference ships no icosphere generator (its `surfaceExamples.py` builds spheres through pygalmesh /
marching cubes); these generators are this package's own and define every synthetic workload:

* ``icosphere(L)`` -- unit icosahedron refined by L rounds of 4-way midpoint subdivision, midpoints
  projected back to the unit sphere and shared per edge. V = 10*4**L + 2 vertices, F = 20*4**L faces,
  faces oriented outward (positive signed volume, the convention of `Surface.surfVolume`,
  base/surfaces.py:1645).
* ``bumpy_ellipsoid(vertices, n_bumps, amplitude, width, seed)`` -- radial Gaussian bumps followed by the
  axis scaling diag(1.2, 1.0, 0.8).
"""
import numpy as np

_PHI = (1.0 + 5.0 ** 0.5) / 2.0

_ICO_FACES = np.array([
    [0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11],
    [1, 5, 9], [5, 11, 4], [11, 10, 2], [10, 7, 6], [7, 1, 8],
    [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9],
    [4, 9, 5], [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]], dtype=np.int64)


def _icosahedron():
    p = _PHI
    v = np.array([[-1, p, 0], [1, p, 0], [-1, -p, 0], [1, -p, 0],
                  [0, -1, p], [0, 1, p], [0, -1, -p], [0, 1, -p],
                  [p, 0, -1], [p, 0, 1], [-p, 0, -1], [-p, 0, 1]], dtype=np.float64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    return v, _ICO_FACES.copy()


def _orient_outward(vertices, faces):
    a, b, c = vertices[faces[:, 0]], vertices[faces[:, 1]], vertices[faces[:, 2]]
    n = np.cross(b - a, c - a)
    centre = (a + b + c) / 3.0
    flip = (n * centre).sum(axis=1) < 0
    faces = faces.copy()
    faces[flip, 1], faces[flip, 2] = faces[flip, 2].copy(), faces[flip, 1].copy()
    return faces


def icosphere(level):
    """Return (vertices (V,3) float64, faces (F,3) int64) of the level-`level` unit icosphere."""
    vertices, faces = _icosahedron()
    verts = [tuple(x) for x in vertices]
    for _ in range(int(level)):
        midpoint = {}
        new_faces = np.empty((faces.shape[0] * 4, 3), dtype=np.int64)

        def mid(i, j):
            key = (i, j) if i < j else (j, i)
            k = midpoint.get(key)
            if k is None:
                m = (np.asarray(verts[i]) + np.asarray(verts[j])) * 0.5
                m /= np.linalg.norm(m)
                k = len(verts)
                verts.append(tuple(m))
                midpoint[key] = k
            return k

        for f, (i, j, k) in enumerate(faces):
            a, b, c = mid(i, j), mid(j, k), mid(k, i)
            new_faces[4 * f + 0] = (i, a, c)
            new_faces[4 * f + 1] = (j, b, a)
            new_faces[4 * f + 2] = (k, c, b)
            new_faces[4 * f + 3] = (a, b, c)
        faces = new_faces
    vertices = np.array(verts, dtype=np.float64)
    faces = _orient_outward(vertices, faces)
    return vertices, faces


def bumpy_ellipsoid(vertices, n_bumps=8, amplitude=0.05, width=0.3, seed=0, axes=(1.2, 1.0, 0.8)):
    """Map unit-sphere vertices to the seeded bumpy ellipsoid.

    r(v) = 1 + A * sum_b exp(-|v - c_b|^2 / (2 w^2)) with c_b = normalize(rng.normal(size=(B, 3))),
    target vertex = diag(axes) (r(v) v), rng = np.random.default_rng(seed).
    """
    rng = np.random.default_rng(seed)
    c = rng.normal(size=(n_bumps, 3))
    c /= np.linalg.norm(c, axis=1, keepdims=True)
    d2 = ((vertices[:, None, :] - c[None, :, :]) ** 2).sum(axis=2)
    r = 1.0 + amplitude * np.exp(-d2 / (2.0 * width ** 2)).sum(axis=1)
    return (vertices * r[:, None]) * np.asarray(axes, dtype=np.float64)[None, :]


def signed_volume(vertices, faces):
    a, b, c = vertices[faces[:, 0]], vertices[faces[:, 1]], vertices[faces[:, 2]]
    return float((a * np.cross(b, c)).sum() / 6.0)


def level_sizes(level):
    """(V, F) of the level-`level` icosphere."""
    return 10 * 4 ** level + 2, 20 * 4 ** level


def registration_pair(level, n_bumps=8, amplitude=0.05, width=0.3, seed=0):
    """Source icosphere and its bumpy-ellipsoid target: (x0, faces, x1)."""
    x0, faces = icosphere(level)
    x1 = bumpy_ellipsoid(x0, n_bumps=n_bumps, amplitude=amplitude, width=width, seed=seed)
    return x0, faces, x1


def smooth_momenta(x, rng, apply_k, sigma_smooth=0.4, sigma_def=0.5, vmax=0.3):
    """Random smooth momenta with a prescribed initial speed: a = K_{sigma_smooth} N(0, 1), rescaled so that the
    velocity K_{sigma_def} a has max norm `vmax`. `apply_k(y, x, a, sigma)` is any Gaussian kernel sum.

    Unnormalised recipes (a = K_s N(0, c^2)) give speeds that grow with the vertex count (7 at 162 vertices, ~400 at
    2,562 for c = 0.1, s = 0.3) and therefore exploding trajectories; the rescaling keeps every level comparable."""
    a = apply_k(x, x, rng.normal(size=x.shape), sigma_smooth)
    v = apply_k(x, x, a, sigma_def)
    return a * (vmax / np.linalg.norm(v, axis=1).max())
