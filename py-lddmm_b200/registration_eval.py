"""Large-mesh registration: seconds to 1e-3 relative energy, learned warm start vs plain, on one GPU.

    python py-lddmm_b200/registration_eval.py [--level 7] [--bumps 32] [--sigma 0.3] [--sigma-dist 0.1]
                                              [--time-step 0.05] [--estar-iters 400] [--fp64-probe-iters 5]

Problem: icosphere at `--level` (level 7: 163,842 vertices, 327,680 faces) -> bumpy ellipsoid with `--bumps` seeded
bumps (amplitude 0.05, width 0.3, seed 0); SecondOrderSurfaceMatching with a Gaussian deformation kernel, unoriented
varifold data term, sigmaError 1, regWeight 1, BFGS.

  1. plain FP32 from zero momentum, run to the BFGS stopping rule (at most `--estar-iters` iterations); its final
     momentum re-evaluated on the FP64 path gives E*, and the first iteration whose FP32 objective is within `--tol`
     of E* gives the plain FP32 iterations and seconds to tolerance (a full FP64 run to the stopping rule is several
     GPU-hours at level 7, so E* comes from the FP32 run and is stated as such);
  2. FP32 from the learned proposal (network trained here on level-4 shot pairs, applied per vertex), stopped at
     E* (1 + tol);
  3. the plain FP64 path timed over `--fp64-probe-iters` BFGS iterations from zero momentum; its seconds to
     tolerance are estimated as (time to the end of its first iteration) + (plain FP32 iterations to tolerance - 1)
     x (its later seconds per iteration) -- the FP64 and FP32 plain runs take the same number of iterations where
     both were run to the end (level 6: 39 and 39).
Prints one JSON line.
"""
import argparse
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import numpy as np  # noqa: E402
import torch  # noqa: E402

from base import learnedProposal as lp  # noqa: E402
from base.kernelFunctions import Kernel  # noqa: E402
from base.surfaceMatching import SecondOrderSurfaceMatching  # noqa: E402
from base.surfaces import Surface  # noqa: E402
from base.syntheticShapes import icosphere, bumpy_ellipsoid  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--level', type=int, default=7)
    ap.add_argument('--bumps', type=int, default=32)
    ap.add_argument('--sigma', type=float, default=0.3)
    ap.add_argument('--sigma-dist', type=float, default=0.1)
    ap.add_argument('--time-step', type=float, default=0.05)
    ap.add_argument('--tol', type=float, default=1e-3)
    ap.add_argument('--estar-iters', type=int, default=400)
    ap.add_argument('--fp64-probe-iters', type=int, default=5, help='at least 2')
    ap.add_argument('--train-pairs', type=int, default=2000)
    ap.add_argument('--train-epochs', type=int, default=20)
    ap.add_argument('--scales', default='0.5,0.75,1.0',
                    help='comma-separated multiples of the proposal tried at the start')
    args = ap.parse_args()
    x0, F = icosphere(args.level)
    x1 = bumpy_ellipsoid(x0, n_bumps=args.bumps, seed=0)
    out = {'problem': f'icosphere L{args.level} ({x0.shape[0]} vertices, {F.shape[0]} faces) -> bumpy ellipsoid '
                      f'({args.bumps} bumps), sigma {args.sigma} / varifold {args.sigma_dist}, '
                      f'T={int(round(1 / args.time_step))}, sigmaError 1, BFGS', 'tol': args.tol}

    def make(dtype, target=None, maxIter=1000):
        K = Kernel(name='gauss', sigma=args.sigma)
        K.pk_dtype = dtype
        opts = dict(maxIter=maxIter, affine='none', regWeight=1.0, KparDiff=K, KparDist=('gauss', args.sigma_dist),
                    sigmaError=1.0, errorType='varifold', pk_dtype=dtype, algorithm='bfgs', timeStep=args.time_step,
                    verb=False, targetObjective=target)
        return SecondOrderSurfaceMatching(Template=Surface(surf=(F, x0)), Target=Surface(surf=(F, x1)), options=opts)

    # 1. plain FP32 to the stopping rule
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    f32 = make('float32', maxIter=args.estar_iters)
    f32.optimizeMatching()
    torch.cuda.synchronize()
    s32_total = time.perf_counter() - t0
    f32.resetPK('float64')
    f32.obj = None
    estar = float(f32.objectiveFun())
    target = estar * (1 + args.tol)
    it32, s32 = None, None
    for i, (e, t) in enumerate(zip(f32.history, f32.times)):
        if e <= target:
            it32, s32 = i + 1, t - t0
            break
    out['plain_fp32'] = {'iters_total': len(f32.history), 'stopped_by_rule': len(f32.history) < args.estar_iters,
                         's_total': s32_total, 'estar_fp64': estar, 'estar_fp32': f32.history[-1],
                         'iters_to_tol': it32, 's_to_tol': s32}
    del f32
    torch.cuda.empty_cache()

    # 2. learned warm start (trained on level-4 shot pairs)
    t0 = time.perf_counter()
    xs, Fs = icosphere(4)
    feats, labels, _, n4 = lp.generate_pairs(xs, Fs, args.train_pairs, seed=0, timeStep=0.1)
    model = lp.MomentumProposal(seed=0)
    hist = lp.train(model, feats, labels, n4, epochs=args.train_epochs, batch_pairs=16, lr=2e-3)
    torch.cuda.synchronize()
    out['proposal'] = {'train_pairs': args.train_pairs, 'epochs': args.train_epochs, 'train_s': time.perf_counter() - t0,
                       'loss_first_last': [hist[0], hist[-1]]}
    del feats, labels
    torch.cuda.empty_cache()
    scales = tuple(float(v) for v in args.scales.split(','))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    fl = make('float32', target=target, maxIter=max(args.estar_iters, 1000))
    used = lp.warm_start(fl, model, scales=scales)
    fl.optimizeMatching()
    torch.cuda.synchronize()
    sl = time.perf_counter() - t0
    fl.resetPK('float64')
    fl.obj = None
    el = float(fl.objectiveFun())
    out['learned_fp32'] = {'iters': len(fl.history), 's_to_tol': sl, 'reached': bool(fl.reached_target),
                           'rel_energy_fp64': (el - estar) / abs(estar), 'proposal_used': used[0],
                           'obj_proposal': used[1], 'obj_zero': used[2], 'scale': used[3]}
    del fl
    torch.cuda.empty_cache()

    # 3. FP64 per-iteration time
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    f64 = make('float64', maxIter=args.fp64_probe_iters)
    f64.optimizeMatching()
    torch.cuda.synchronize()
    s64 = time.perf_counter() - t0
    # f64.times[i] closes iteration i + 1 (the last entry repeats the final iteration when maxIter ends the run)
    first = f64.times[0] - t0
    k = args.fp64_probe_iters
    per_it = (f64.times[k - 1] - f64.times[0]) / (k - 1)
    out['plain_fp64_probe'] = {'iters': k, 's': s64, 's_first_iter': first, 's_per_iter': per_it,
                               'history': f64.history[:k]}
    if it32 is not None:
        est = first + per_it * (it32 - 1)
        out['plain_fp64_s_to_tol_estimate'] = est
        out['speedup_learned_vs_plain_fp64_estimate'] = est / sl
        out['speedup_plain_fp32_vs_plain_fp64_estimate'] = est / s32
    print(json.dumps(out), flush=True)


if __name__ == '__main__':
    main()
