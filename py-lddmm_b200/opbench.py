"""Per-operator timing of the hot kernels on synthetic icosphere inputs.

    python py-lddmm_b200/opbench.py [--level 6] [--ops all] [--precision fp32|fp64] [--reps 10] [--warmup 3]
                                    [--kernel gauss|laplacian:<order>]

For every operator: device time per call (CUDA events on the launching stream, after warm-up), pair evaluations
per second, FP32 lane-ops per second from the per-pair operation counts of the kernel, and the fraction of the
FP32 pipe peak (SMs x 128 lanes x max SM clock); the operation counts are those of the Gaussian kernel, so with
--kernel laplacian only times and pairs/s are reported. One JSON line per operator. Used for the ncu captures in
profiles/ (run it with --reps 1 --warmup 0 under ncu to capture one launch per operator).
"""
import argparse
import ctypes
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import numpy as np  # noqa: E402
import torch  # noqa: E402

from base import _native as nat  # noqa: E402
from base.surfaceDistances import vertex_face_table  # noqa: E402
from base.syntheticShapes import icosphere, bumpy_ellipsoid  # noqa: E402

# FP32 lane-ops and SFU ops per pair of each kernel (packed instructions counted per lane); applyK, the
# second-order step and the varifold energy and gradient: their expanded-distance form (blocks whose radius is too
# large for it take the difference form: 9, 16, 12 and 22)
OPS = {'applyK': (6, 1), 'applyDiffKT_lddmm': (16, 1), 'applyDDiffK11and12': (23, 1), 'applyDiffK1and2': (16, 1),
       'so_step': (14, 1), 'so_adjoint_step': (37, 1), 'fo_adjoint_step': (19, 1), 'varifold_energy': (9, 1),
       'varifold_gradient': (19, 1)}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--level', type=int, default=6)
    ap.add_argument('--ops', default='all')
    ap.add_argument('--precision', default='fp32', choices=['fp32', 'fp64'])
    ap.add_argument('--reps', type=int, default=10)
    ap.add_argument('--warmup', type=int, default=3)
    ap.add_argument('--sigma', type=float, default=0.5)
    ap.add_argument('--sigma-dist', type=float, default=0.2)
    ap.add_argument('--kernel', default='gauss', help="deformation kernel: 'gauss' or 'laplacian:<order>'")
    args = ap.parse_args()
    kern = nat.KERNEL_GAUSS if args.kernel == 'gauss' else nat.KERNEL_LAPLACIAN0 + int(args.kernel.split(':')[1])
    prec = nat.FP32C if args.precision == 'fp32' else nat.FP64
    lib = nat.lib()
    x, F = icosphere(args.level)
    x1 = bumpy_ellipsoid(x, seed=0)
    n, nf = x.shape[0], F.shape[0]
    rng = np.random.default_rng(0)
    X, X1 = torch.from_numpy(x).cuda(), torch.from_numpy(x1).cuda()
    FF = torch.from_numpy(F).cuda()
    A = torch.from_numpy(rng.normal(0, 0.01, x.shape)).cuda()
    P = torch.from_numpy(rng.normal(size=x.shape)).cuda()
    Q = torch.from_numpy(rng.normal(0, 0.1, x.shape)).cuda()
    o1, o2 = torch.empty_like(X), torch.empty_like(X)
    dat = torch.empty_like(X)
    E = torch.zeros(2, dtype=torch.float64, device='cuda')
    off, items = vertex_face_table(F, n)
    o = nat.origin_arg(nat.centroid(X))
    ws, wsb = nat.workspace(n, n, prec)
    sws, swsb = nat.surface_workspace(nf, nf, prec)
    st = nat.stream_ptr()
    p = nat.ptr
    s, sd = args.sigma, args.sigma_dist

    def ok(rc):
        if rc != 0:
            raise RuntimeError(lib.lddmm_status_string(rc).decode())

    calls = {
        'applyK': (lambda: ok(lib.lddmm_apply_k(p(X), n, p(X), p(A), n, s, kern, o, p(o1), prec, ws, wsb, st))),
        'applyDiffKT_lddmm': (lambda: ok(lib.lddmm_apply_diff_kt(p(X), n, p(X), p(P), p(A), n, s, kern, 2, 1.0, o,
                                                                   p(o1), prec, ws, wsb, st))),
        'applyDDiffK11and12': (lambda: ok(lib.lddmm_apply_ddiff_k11and12(p(X), p(A), p(A), p(Q), n, s, kern, o, p(o1),
                                                                         prec, ws, wsb, st))),
        'applyDiffK1and2': (lambda: ok(lib.lddmm_apply_diff_k1and2(p(X), p(Q), p(A), n, s, kern, o, p(o1), prec, ws,
                                                                   wsb, st))),
        'so_step': (lambda: ok(lib.lddmm_second_order_step(p(X), p(A), n, s, kern, 0.05, o, p(o1), p(o2), prec, ws,
                                                           wsb, st))),
        'so_adjoint_step': (lambda: ok(lib.lddmm_second_order_adjoint_step(p(X), p(A), p(P), p(Q), n, s, kern, 0.05,
                                                                           o, p(o1), p(o2), prec, ws, wsb, st))),
        'varifold_energy': (lambda: ok(lib.lddmm_surface_energy(0, p(X), n, p(FF), nf, None, p(X1), n, p(FF), nf, None,
                                                                sd, o, 0, p(E), prec, sws, swsb, st))),
        'varifold_gradient': (lambda: ok(lib.lddmm_surface_gradient(0, p(X), n, p(FF), nf, None, p(off), p(items),
                                                                    p(X1), n, p(FF), nf, None, sd, o, p(o1), None,
                                                                    prec, sws, swsb, st))),
    }
    # the first-order adjoint entry point runs T steps: time one step with a 2-state trajectory
    XT = torch.stack([X, X])
    AT = A.unsqueeze(0).contiguous()
    PXT = torch.empty_like(XT)
    calls['fo_adjoint_step'] = (lambda: ok(lib.lddmm_first_order_gradient(p(XT), p(AT), n, 1, s, kern, 1.0, p(P), 1,
                                                                          o, p(PXT), p(dat), prec, ws, wsb, st)))
    pairs = {k: float(n) * n for k in calls}
    pairs['varifold_energy'] = float(nf) * 2 * nf
    pairs['varifold_gradient'] = float(nf) * 2 * nf
    props = torch.cuda.get_device_properties(0)
    sm_clock = float(os.environ.get('SM_MHZ', '1965'))
    peak = props.multi_processor_count * 128 * sm_clock * 1e6
    names = list(calls) if args.ops == 'all' else args.ops.split(',')
    for name in names:
        fn = calls[name]
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / max(args.reps, 1)
        pps = pairs[name] / (ms * 1e-3)
        fp32, sfu = OPS[name]
        gauss = kern == nat.KERNEL_GAUSS or name.startswith('varifold')   # the op counts are the Gaussian ones
        line = {'op': name, 'kernel': args.kernel if not name.startswith('varifold') else 'gauss',
                'level': args.level, 'precision': args.precision, 'ms': round(ms, 4), 'pairs_per_s': pps,
                'fp32_lane_ops_per_s': pps * fp32 if gauss else None,
                'frac_fp32_peak': pps * fp32 / peak if args.precision == 'fp32' and gauss else None,
                'frac_sfu_peak': pps * sfu / (props.multi_processor_count * 16 * sm_clock * 1e6) if gauss else None}
        print(json.dumps(line), flush=True)


if __name__ == '__main__':
    main()
