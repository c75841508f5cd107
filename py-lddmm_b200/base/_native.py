"""ctypes binding of the sm_100a C-ABI library `lib/liblddmm_b200.so` (declared in include/lddmm_b200.h).

PyTorch supplies device memory and the current CUDA stream; every computation runs in the library.
There is no CPU fallback: when the library or a CUDA device is missing, `lib()` raises.
"""
import ctypes
import os
import threading

import numpy as np
import torch

_HERE = os.path.dirname(os.path.abspath(__file__))
# the in-tree build; LDDMM_B200_LIB names another build of the same library (e.g. one compiled with other tuning
# macros) to load instead
LIB_PATH = os.environ.get('LDDMM_B200_LIB') or os.path.join(os.path.dirname(_HERE), 'lib', 'liblddmm_b200.so')

FP32C = 0
FP64 = 1
KERNEL_GAUSS = 0
KERNEL_LAPLACIAN0 = 16     # + order (0..4)
DATA_VARIFOLD, DATA_CURRENT, DATA_MEASURE = 0, 1, 2

_i64, _f64, _int, _sz, _vp = ctypes.c_int64, ctypes.c_double, ctypes.c_int, ctypes.c_size_t, ctypes.c_void_p
_dp = ctypes.c_void_p          # device pointer
_hp = ctypes.POINTER(ctypes.c_double)  # host pointer (origin)

# name -> argtypes (restype int unless listed in _RESTYPES)
SIGNATURES = {
    'lddmm_version': [],
    'lddmm_status_string': [_int],
    'lddmm_workspace_bytes': [_i64, _i64, _int],
    'lddmm_surface_workspace_bytes': [_i64, _i64, _int],
    'lddmm_apply_k': [_dp, _i64, _dp, _dp, _i64, _f64, _int, _hp, _dp, _int, _vp, _sz, _vp],
    'lddmm_apply_diff_kt': [_dp, _i64, _dp, _dp, _dp, _i64, _f64, _int, _int, _f64, _hp, _dp, _int, _vp, _sz, _vp],
    'lddmm_apply_ddiff_k11and12': [_dp, _dp, _dp, _dp, _i64, _f64, _int, _hp, _dp, _int, _vp, _sz, _vp],
    'lddmm_apply_diff_k1and2': [_dp, _dp, _dp, _i64, _f64, _int, _hp, _dp, _int, _vp, _sz, _vp],
    'lddmm_apply_divergence': [_dp, _i64, _dp, _dp, _i64, _f64, _int, _hp, _dp, _int, _vp, _sz, _vp],
    'lddmm_apply_k_tensor': [_dp, _i64, _dp, _i64, _dp, _dp, _dp, _dp, _f64, _hp, _dp, _int, _vp, _sz, _vp],
    'lddmm_apply_k_static': [_dp, _i64, _dp, _dp, _i64, _f64, _hp, _dp, _int, _vp],
    'lddmm_apply_k_mat': [_dp, _i64, _dp, _i64, _dp, _i64, _f64, _dp, _vp],
    'lddmm_apply_diff_k_mat': [_dp, _i64, _dp, _i64, _dp, _f64, _dp, _vp],
    'lddmm_second_order_step': [_dp, _dp, _i64, _f64, _int, _f64, _hp, _dp, _dp, _int, _vp, _sz, _vp],
    'lddmm_second_order_shoot': [_dp, _dp, _i64, _i64, _f64, _int, _f64, _hp, _dp, _dp, _int, _vp, _sz, _vp],
    'lddmm_second_order_step_rows': [_dp, _dp, _i64, _i64, _i64, _f64, _int, _f64, _hp, _dp, _dp, _int, _vp, _sz,
                                     _vp],
    'lddmm_second_order_adjoint_step_rows': [_dp, _dp, _dp, _dp, _i64, _i64, _i64, _f64, _int, _f64, _hp, _dp, _dp,
                                             _int, _vp, _sz, _vp],
    'lddmm_second_order_adjoint_step': [_dp, _dp, _dp, _dp, _i64, _f64, _int, _f64, _hp, _dp, _dp, _int, _vp, _sz,
                                        _vp],
    'lddmm_second_order_gradient': [_dp, _dp, _i64, _i64, _f64, _int, _f64, _dp, _dp, _hp, _dp, _dp, _dp, _int, _vp,
                                    _sz, _vp],
    'lddmm_first_order_shoot': [_dp, _dp, _i64, _i64, _f64, _int, _f64, _hp, _dp, _dp, _int, _vp, _sz, _vp],
    'lddmm_first_order_gradient': [_dp, _dp, _i64, _i64, _f64, _int, _f64, _dp, _int, _hp, _dp, _dp, _int, _vp, _sz,
                                   _vp],
    'lddmm_surface_energy': [_int, _dp, _i64, _dp, _i64, _dp, _dp, _i64, _dp, _i64, _dp, _f64, _hp, _int, _dp, _int,
                             _vp, _sz, _vp],
    'lddmm_surface_gradient': [_int, _dp, _i64, _dp, _i64, _dp, _dp, _dp, _dp, _i64, _dp, _i64, _dp, _f64, _hp, _dp,
                               _dp, _int, _vp, _sz, _vp],
    'lddmm_vertex_face_table': [_vp, _i64, _i64, _vp, _vp],
    'lddmm_bf16_gemm': [_int, _int, _int, _i64, _i64, _i64, _dp, _dp, _dp, _dp, _dp, _int, _dp, _sz, _vp],
    'lddmm_bf16_colsum': [_dp, _i64, _i64, _dp, _dp, _sz, _vp],
    'lddmm_mse_grad': [_dp, _i64, _i64, _dp, _i64, _i64, ctypes.c_float, _dp, _dp, _vp],
    'lddmm_adam_step': [_dp, _dp, _dp, _dp, _dp, _i64, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                        ctypes.c_float, _i64, ctypes.c_float, _vp],
    'lddmm_nearest_displacement': [_dp, _i64, _dp, _i64, _dp, _vp],
    'lddmm_lbfgs_direction': [_vp, _vp, _int, _dp, _i64, _dp, _vp],
}
LBFGS_MAX_PAIRS = 64        # LDDMM_LBFGS_MAX_PAIRS of the header
_RESTYPES = {'lddmm_version': ctypes.c_char_p, 'lddmm_status_string': ctypes.c_char_p,
             'lddmm_workspace_bytes': ctypes.c_size_t, 'lddmm_surface_workspace_bytes': ctypes.c_size_t}

_lib = None
_lock = threading.Lock()
_PINNED_MIN_BYTES = 1 << 16   # host <-> device copies at least this large go through page-locked staging


class LddmmError(RuntimeError):
    pass


def load_library(path=LIB_PATH):
    """Load the shared library and declare every entry point (no device needed)."""
    if not os.path.exists(path):
        raise LddmmError(f'lddmm_b200 native library not found at {path}; build it with py-lddmm_b200/build.py')
    lib = ctypes.CDLL(path)
    for name, args in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = _RESTYPES.get(name, ctypes.c_int)
    return lib


def lib():
    """The loaded library; raises if it is missing or no CUDA device is available (no CPU fallback)."""
    global _lib
    if _lib is None:
        with _lock:
            if _lib is None:
                if not torch.cuda.is_available():
                    raise LddmmError('lddmm_b200 needs a CUDA device (sm_100a); none is available')
                _lib = load_library()
    return _lib


def kernel_code(K):
    """The library's kernel-family argument for a Kernel: 0 (Gaussian) or 16 + order ('laplacian')."""
    name = getattr(K, 'name', 'gauss')
    if name in ('gauss', 'gaussian'):
        return KERNEL_GAUSS
    if name == 'laplacian':
        return KERNEL_LAPLACIAN0 + int(K.order)
    raise NotImplementedError(f"lddmm_b200 implements the 'gauss' and 'laplacian' kernels (got '{name}')")


def check(status, what=''):
    if status != 0:
        msg = lib().lddmm_status_string(status).decode()
        raise LddmmError(f'{what}: lddmm status {status} ({msg})')


def stream_ptr():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else ctypes.c_void_p(0)


def origin_arg(origin):
    if origin is None:
        return None
    o = (ctypes.c_double * 3)(*[float(v) for v in origin])
    return ctypes.cast(o, _hp)


class Workspace:
    """Per-device scratch buffer grown on demand (torch caching allocator). A buffer that is outgrown is retired,
    not freed: a caller that took its pointer before another request grew the workspace keeps valid memory (the
    retired buffers add up to less than the current one, sizes being powers of two)."""

    def __init__(self):
        self._bufs = {}
        self._retired = {}

    def get(self, nbytes, device=None):
        dev = torch.device('cuda', torch.cuda.current_device() if device is None else device)
        buf = self._bufs.get(dev.index)
        if buf is None or buf.numel() < nbytes:
            size = max(int(nbytes), 1 << 20)
            size = 1 << (size - 1).bit_length()
            if buf is not None:
                self._retired.setdefault(dev.index, []).append(buf)
            buf = torch.empty(size, dtype=torch.uint8, device=dev)
            self._bufs[dev.index] = buf
        return buf


WORKSPACE = Workspace()


_WS_BYTES = {}   # (entry, n, m, precision, device) -> bytes: the library's answer depends on nothing else


def _ws_bytes(entry, n, m, precision):
    key = (entry, int(n), int(m), int(precision), torch.cuda.current_device())
    nb = _WS_BYTES.get(key)
    if nb is None:
        nb = _WS_BYTES[key] = getattr(lib(), entry)(key[1], key[2], key[3])
    return nb


def workspace(n, m, precision=FP32C):
    buf = WORKSPACE.get(_ws_bytes('lddmm_workspace_bytes', n, m, precision))
    return ctypes.c_void_p(buf.data_ptr()), ctypes.c_size_t(buf.numel())


def surface_workspace(nf, nf1, precision=FP32C):
    buf = WORKSPACE.get(_ws_bytes('lddmm_surface_workspace_bytes', nf, nf1, precision))
    return ctypes.c_void_p(buf.data_ptr()), ctypes.c_size_t(buf.numel())


def as_device(a, device=None, dtype=torch.float64):
    """numpy / torch -> contiguous CUDA tensor of `dtype` (no copy when already so)."""
    if isinstance(a, torch.Tensor):
        t = a
        if not t.is_cuda:
            t = t.to(device='cuda' if device is None else device, non_blocking=False)
        if t.dtype != dtype:
            t = t.to(dtype)
        return t.contiguous()
    arr = np.ascontiguousarray(np.asarray(a), dtype=np.float64 if dtype == torch.float64 else None)
    t = torch.from_numpy(arr)
    if dtype != t.dtype:
        t = t.to(dtype)
    if t.numel() * t.element_size() >= _PINNED_MIN_BYTES:
        # staged through page-locked memory (torch's caching host allocator) and copied asynchronously on the
        # current stream; the staging block is not reused before the copy has completed
        return t.pin_memory().to(device='cuda' if device is None else device, non_blocking=True)
    return t.to(device='cuda' if device is None else device)


def to_host(t):
    """Device tensor -> new numpy array, read back through page-locked memory for large results."""
    if t.numel() * t.element_size() < _PINNED_MIN_BYTES:
        return t.cpu().numpy()
    h = torch.empty(t.shape, dtype=t.dtype, pin_memory=True)
    h.copy_(t, non_blocking=True)
    torch.cuda.current_stream().synchronize()
    return h.numpy()


def centroid(t):
    """Centre used as the FP32 origin (results are translation invariant). Host arrays are averaged on the host;
    device tensors with one reduction (and one synchronisation)."""
    if not isinstance(t, torch.Tensor):
        a = np.asarray(t, dtype=np.float64).reshape(-1, 3)
        # ones @ a (one BLAS gemv) instead of a.mean(axis=0), whose strided reduction is ~20x slower for (N,3)
        return None if a.size == 0 else (np.ones(a.shape[0]) @ a / a.shape[0]).tolist()
    if t.numel() == 0:
        return None
    return t.reshape(-1, 3).mean(dim=0).tolist()
