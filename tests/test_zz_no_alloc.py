"""lddmm_apply_k_static: the allocation-free K(y, x) a, for callers that cannot allocate device memory when they
call the library (a fixed device-memory budget, a plugin host without an allocator, or a latency-critical path
where cudaMalloc could synchronise the device).

The entry point is called through the C ABI (ctypes) twice in a row -- the second call reuses the scratch array
that the first call left filled -- and each result is compared with the workspace-based lddmm_apply_k on the same
inputs, within the tolerance of the other kernel-sum tests, for both arithmetic paths (FP32 compensated and FP64,
each with its own launch plan in the shared array). One case sits near the array's capacity: 226,301 targets
against a million sources is the request with the largest scratch on a B200 (4 partial slots per target, 20.7 MiB
of the 32 MiB). This file is collected last so that a run stopping at the first failure has already run every other
test; it also passes alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = {0: 2e-5, 1: 1e-12}   # relative L2 error by precision (FP32C, FP64), as in tests/test_gpu_kernels.py


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _run(lib, nat, torch, Y, X, A, sigma, static, precision):
    out = torch.empty((Y.shape[0], 3), dtype=torch.float64, device='cuda')
    o = nat.origin_arg(nat.centroid(X))
    if static:
        rc = lib.lddmm_apply_k_static(nat.ptr(Y), Y.shape[0], nat.ptr(X), nat.ptr(A), X.shape[0], sigma, o,
                                      nat.ptr(out), precision, nat.stream_ptr())
    else:
        ws, wsb = nat.workspace(Y.shape[0], X.shape[0], precision)
        rc = lib.lddmm_apply_k(nat.ptr(Y), Y.shape[0], nat.ptr(X), nat.ptr(A), X.shape[0], sigma, nat.KERNEL_GAUSS, o,
                               nat.ptr(out), precision, ws, wsb, nat.stream_ptr())
    assert rc == 0, lib.lddmm_status_string(rc)
    torch.cuda.synchronize()
    return out.cpu().numpy()


@pytest.mark.parametrize('precision', [0, 1], ids=['fp32c', 'fp64'])
def test_static_scratch_matches_workspace_entry_point_twice(precision):
    import torch
    from base import _native as nat
    lib = nat.lib()
    rng = np.random.default_rng(11)
    cases = [(40962, 40962, 0.25), (3000, 20000, 0.5)]     # two calls in a row, different sizes
    for n, m, sigma in cases:
        Y = torch.from_numpy(rng.normal(size=(n, 3))).cuda()
        X = torch.from_numpy(rng.normal(size=(m, 3))).cuda()
        A = torch.from_numpy(rng.normal(size=(m, 3))).cuda()
        ref = _run(lib, nat, torch, Y, X, A, sigma, False, precision)
        got = _run(lib, nat, torch, Y, X, A, sigma, True, precision)
        assert _rel(got, ref) < TOL[precision], (n, m, _rel(got, ref))


@pytest.mark.parametrize('precision,n,m', [(0, 226301, 1000000), (1, 262144, 600000)], ids=['fp32c', 'fp64'])
def test_static_scratch_near_capacity(precision, n, m):
    """The largest scratch request on a B200 (FP32: 4 partial slots for each of 226,301 targets, 20.7 MiB) and the
    largest target count for the FP64 plan, each compared with the workspace entry point, twice in a row."""
    import torch
    from base import _native as nat
    lib = nat.lib()
    rng = np.random.default_rng(12)
    Y = torch.from_numpy(rng.uniform(-1, 1, size=(n, 3))).cuda()
    X = torch.from_numpy(rng.uniform(-1, 1, size=(m, 3))).cuda()
    A = torch.from_numpy(rng.normal(size=(m, 3))).cuda()
    ref = _run(lib, nat, torch, Y, X, A, 0.05, False, precision)
    for _ in range(2):
        got = _run(lib, nat, torch, Y, X, A, 0.05, True, precision)
        assert _rel(got, ref) < TOL[precision], (n, m, _rel(got, ref))


def test_static_scratch_rejects_oversize_before_launch():
    import torch
    from base import _native as nat
    lib = nat.lib()
    n = 262145                      # one target over the stated maximum; buffers are real so nothing could fault
    Y = torch.zeros((n, 3), dtype=torch.float64, device='cuda')
    A = torch.zeros((16, 3), dtype=torch.float64, device='cuda')
    out = torch.full((n, 3), 7.0, dtype=torch.float64, device='cuda')
    rc = lib.lddmm_apply_k_static(nat.ptr(Y), n, nat.ptr(A), nat.ptr(A), 16, 0.5, None, nat.ptr(out), nat.FP32C,
                                  nat.stream_ptr())
    assert rc == 4     # LDDMM_ERR_WORKSPACE
    torch.cuda.synchronize()
    assert bool((out == 7.0).all())
