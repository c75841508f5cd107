"""Mesh I/O on real meshes of the reference's test data (tests/golden/meshes, copied by make_mesh_fixtures.py):
the OBJ and legacy-VTK readers, a VTK write/read round trip, and the vertex areas of the result descriptors."""
import os

import numpy as np

from conftest import GOLDEN

MESHES = os.path.join(GOLDEN, 'meshes')


def _obj_counts(path):
    nv = nf = 0
    for line in open(path):
        if line.startswith('v '):
            nv += 1
        elif line.startswith('f '):
            nf += 1
    return nv, nf


def test_read_obj_real_mesh():
    from base.surfaces import Surface
    path = os.path.join(MESHES, 'spot_triangulated_reduced.obj')
    s = Surface(surf=path)
    nv, nf = _obj_counts(path)
    assert s.vertices.shape == (nv, 3) and s.faces.shape == (nf, 3)
    assert s.faces.min() == 0 and s.faces.max() == nv - 1
    # coordinates are the file's values rounded to single precision, as vtk's reader stores them
    first = [float(t) for t in next(ln for ln in open(path) if ln.startswith('v ')).split()[1:4]]
    assert np.array_equal(s.vertices[0], np.float32(first).astype(np.float64))
    # a closed, consistently oriented surface: every edge is shared by two faces in opposite directions
    e = np.concatenate([s.faces[:, [0, 1]], s.faces[:, [1, 2]], s.faces[:, [2, 0]]])
    fwd = {tuple(x) for x in e}
    assert all((b, a) in fwd for a, b in fwd)
    assert abs(s.surfVolume()) > 0 and s.surfArea() > 0


def test_read_vtk_real_mesh_and_round_trip(tmp_path):
    from base.surfaces import Surface, read_vtk_ascii
    path = os.path.join(MESHES, 'Hippo.vtk')
    s = Surface(surf=path)
    assert s.vertices.shape == (1001, 3) and s.faces.shape == (1998, 3)
    assert s.faces.min() == 0 and s.faces.max() == 1000
    assert np.all(s.weights == 1)
    out = os.path.join(tmp_path, 'hippo_copy.vtk')
    s.saveVTK(out)
    f2, v2 = read_vtk_ascii(out)        # written as double: read back exactly
    assert np.array_equal(f2, s.faces) and np.array_equal(v2, s.vertices)
    c = s.centers
    assert np.allclose(c, (s.vertices[s.faces[:, 0]] + s.vertices[s.faces[:, 1]] + s.vertices[s.faces[:, 2]]) / 3)


def test_vertex_areas_sum_to_surface_area():
    from base.surfaces import Surface
    for name in ('Hippo.vtk', 'spot_triangulated_reduced.obj'):
        s = Surface(surf=os.path.join(MESHES, name))
        for simple in (True, False):
            av, af = s.computeVertexArea(simpleMethod=simple)
            assert np.isclose(av.sum(), af.sum(), rtol=1e-12)
            assert np.isclose(af.sum(), s.surfArea(), rtol=1e-12)
            assert np.all(av > 0)


def test_mixed_vertex_area_rule_on_two_triangles():
    """One acute and one obtuse triangle, areas by hand from the rule's definition."""
    from base.surfaces import Surface
    v = np.array([[0., 0, 0], [1, 0, 0], [0, 1, 0], [3, 3, 0]])
    s = Surface(surf=(np.array([[0, 1, 2]]), v[:3]))
    av, af = s.computeVertexArea()
    # right angle at vertex 0 (not obtuse): corners get (|e|^2 cot + |e'|^2 cot') / 8
    assert np.allclose(av, [0.25, 0.125, 0.125]) and np.isclose(af[0], 0.5)
    s2 = Surface(surf=(np.array([[1, 3, 2]]), v))
    av2, af2 = s2.computeVertexArea()
    assert np.isclose(av2.sum(), af2[0]) and np.all(av2[[1, 2, 3]] > 0) and av2[0] == 0
