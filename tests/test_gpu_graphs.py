"""The C-ABI entry points of a registration step run inside a captured CUDA graph: kernel sums, geodesic shooting,
its adjoint sweep and the varifold gradient are captured once (torch.cuda.graph, workspace and topology tables
prepared beforehand), then replayed on new inputs written into the captured buffers; every replay equals the eager
calls on the same inputs bit for bit (same kernels, same launch plans, fixed-order reductions)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_registration_step_replays_in_a_cuda_graph():
    import torch
    from base import _native as nat
    from base.surfaceDistances import vertex_face_table
    from base.syntheticShapes import icosphere, bumpy_ellipsoid
    lib = nat.lib()
    x0, F = icosphere(4)
    x1 = bumpy_ellipsoid(x0, seed=0)
    n, nf, T, dt, sigma, sd = x0.shape[0], F.shape[0], 10, 0.1, 0.5, 0.3
    X0 = torch.from_numpy(x0).cuda()
    X1 = torch.from_numpy(x1).cuda()
    FF = torch.from_numpy(np.ascontiguousarray(F, dtype=np.int64)).cuda()
    off, items = vertex_face_table(F, n)
    A0 = torch.zeros_like(X0)
    xt = torch.empty((T + 1, n, 3), dtype=torch.float64, device='cuda')
    at, pxt, pat = torch.empty_like(xt), torch.empty_like(xt), torch.empty_like(xt)
    ka, px1, da0 = torch.empty_like(X0), torch.empty_like(X0), torch.empty_like(X0)
    pa1 = torch.zeros_like(X0)
    o = nat.origin_arg(nat.centroid(X0))
    p = nat.ptr
    # private scratch of the exact sizes the library asks for, allocated before capture
    wsb = lib.lddmm_workspace_bytes(n, n, nat.FP32C)
    swsb = lib.lddmm_surface_workspace_bytes(nf, nf, nat.FP32C)
    W = torch.empty(wsb, dtype=torch.uint8, device='cuda')
    SW = torch.empty(swsb, dtype=torch.uint8, device='cuda')
    ws, sws = p(W), p(SW)

    def step():
        st = nat.stream_ptr()
        nat.check(lib.lddmm_apply_k(p(X0), n, p(X0), p(A0), n, sigma, nat.KERNEL_GAUSS, o, p(ka), nat.FP32C, ws, wsb,
                                    st), 'apply_k')
        nat.check(lib.lddmm_second_order_shoot(p(X0), p(A0), n, T, sigma, nat.KERNEL_GAUSS, dt, o, p(xt), p(at),
                                               nat.FP32C, ws, wsb, st), 'shoot')
        nat.check(lib.lddmm_surface_gradient(nat.DATA_VARIFOLD, p(xt[T]), n, p(FF), nf, None, p(off), p(items),
                                             p(X1), n, p(FF), nf, None, sd, o, p(px1), None, nat.FP32C, sws, swsb,
                                             st), 'varifold gradient')
        nat.check(lib.lddmm_second_order_gradient(p(xt), p(at), n, T, sigma, nat.KERNEL_GAUSS, dt, p(px1), p(pa1), o,
                                                  p(pxt), p(pat), p(da0), nat.FP32C, ws, wsb, st), 'adjoint')

    def outputs():
        return [t.clone() for t in (ka, xt, at, px1, pxt, pat, da0)]

    rng = np.random.default_rng(0)
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        A0.copy_(torch.from_numpy(rng.normal(0.0, 0.002, x0.shape)))
        step()                      # eager warm-up: launch plans and occupancy queries are cached here
    torch.cuda.current_stream().wait_stream(side)
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        step()
    for trial in range(3):
        A0.copy_(torch.from_numpy(rng.normal(0.0, 0.002, x0.shape)))
        g.replay()
        torch.cuda.synchronize()
        replayed = outputs()
        step()
        torch.cuda.synchronize()
        eager = outputs()
        for k, (r, e) in enumerate(zip(replayed, eager)):
            assert torch.equal(r, e), (trial, k)
        assert float(da0.abs().max()) > 0.0
    del g
