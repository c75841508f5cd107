"""The C-ABI library loads without a GPU and exports every entry point that include/lddmm_b200.h declares."""
import ctypes
import os
import re

from conftest import REPO

HEADER = os.path.join(REPO, 'include', 'lddmm_b200.h')


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r'/\*.*?\*/', '', src, flags=re.S)
    names = re.findall(r'\b(lddmm_[a-z0-9_]+)\s*\(', src)
    return sorted(set(names))


def test_header_declares_entry_points():
    names = declared_functions()
    for must in ('lddmm_apply_k', 'lddmm_apply_diff_kt', 'lddmm_apply_ddiff_k11and12', 'lddmm_apply_diff_k1and2',
                 'lddmm_apply_k_tensor', 'lddmm_second_order_shoot', 'lddmm_second_order_gradient',
                 'lddmm_first_order_shoot', 'lddmm_first_order_gradient', 'lddmm_surface_energy',
                 'lddmm_surface_gradient', 'lddmm_workspace_bytes'):
        assert must in names


def test_library_exports_every_declared_symbol():
    from base import _native as nat
    lib = nat.load_library()
    for name in declared_functions():
        assert hasattr(lib, name), name
    # every declared function has a ctypes signature in the binding, and vice versa
    assert set(declared_functions()) == set(nat.SIGNATURES)


def test_host_only_entry_points():
    """Calls that need no device: version, status strings, argument validation before any launch."""
    from base import _native as nat
    lib = nat.load_library()
    assert b'sm_100a' in lib.lddmm_version()
    assert lib.lddmm_status_string(0) == b'ok'
    assert lib.lddmm_status_string(1) == b'invalid argument'
    # negative sizes and non-positive sigma are rejected before touching the device
    null = ctypes.c_void_p(0)
    assert lib.lddmm_apply_k(null, -1, null, null, 0, 0.5, 0, None, null, 0, null, 0, null) == 1
    assert lib.lddmm_apply_k(null, 0, null, null, 0, -0.5, 0, None, null, 0, null, 0, null) == 1
    assert lib.lddmm_apply_k(null, 0, null, null, 0, 0.5, 7, None, null, 0, null, 0, null) == 1     # unknown family
    assert lib.lddmm_apply_k(null, 0, null, null, 0, 0.5, 21, None, null, 0, null, 0, null) == 1    # order 5
    assert lib.lddmm_apply_diff_kt(null, 4, null, null, null, 5, 0.5, 0, 2, 1.0, None, null, 0, null, 0, null) == 1
    assert lib.lddmm_second_order_shoot(null, null, 0, 1, 0.5, 3, 0.1, None, null, null, 0, null, 0, null) == 1
    assert lib.lddmm_workspace_bytes(10, 10, 7) == 0
    # the L-BFGS direction takes 1..64 stored pairs
    assert lib.lddmm_lbfgs_direction(null, null, 0, null, 10, null, null) == 1
    assert lib.lddmm_lbfgs_direction(null, null, 65, null, 10, null, null) == 1


def test_vertex_face_table_host():
    import numpy as np
    from base import _native as nat
    from base.syntheticShapes import icosphere
    lib = nat.load_library()
    v, f = icosphere(2)
    f = np.ascontiguousarray(f, dtype=np.int64)
    off = np.zeros(v.shape[0] + 1, dtype=np.int32)
    items = np.zeros(3 * f.shape[0], dtype=np.int32)
    assert lib.lddmm_vertex_face_table(f.ctypes.data, f.shape[0], v.shape[0], off.ctypes.data, items.ctypes.data) == 0
    assert off[-1] == 3 * f.shape[0]
    for vi in range(v.shape[0]):
        its = items[off[vi]:off[vi + 1]]
        assert np.all(np.diff(its) > 0)
        assert np.all(f.ravel()[its] == vi)
    bad = f.copy()
    bad[0, 0] = v.shape[0] + 5
    assert lib.lddmm_vertex_face_table(bad.ctypes.data, bad.shape[0], v.shape[0], off.ctypes.data,
                                       items.ctypes.data) == 1
