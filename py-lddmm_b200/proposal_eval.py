"""Held-out evaluation of the learned momentum proposal: iterations and seconds to tolerance, plain vs learned.

    python py-lddmm_b200/proposal_eval.py [--pairs 20000] [--heldout 2000] [--eval 100] [--epochs 8]

Training set: `--pairs` source/target pairs generated by shooting random smooth normal momenta from the level-4
icosphere (Gaussian sigma 0.5, T = 10; `learnedProposal.generate_pairs`); the last `--heldout` pairs are held out
and never trained on. The network is trained on the rest with the library's BF16 kernels.

Evaluation on the first `--eval` held-out pairs, each registered as a surface (SecondOrderSurfaceMatching, Gaussian
sigma 0.5, unoriented varifold sigma 0.3, sigmaError 1, T = 10, BFGS):
  1. plain FP64 from zero momentum, run to the BFGS stopping rule: its last objective is the pair's E*, and the
     first iteration whose objective is within `--tol` of E* gives the plain FP64 iterations / seconds;
  2. plain FP32 from zero momentum, stopped at E* (1 + tol);
  3. FP32 from the learned proposal (zero-momentum fallback when the proposal does not lower the objective),
     stopped at E* (1 + tol).
Prints one JSON line per evaluated pair (with --verbose) and a summary line: mean / median iterations and seconds
of the three runs and the fraction of pairs on which the proposal was used.
"""
import argparse
import json
import os
import statistics
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
from base.syntheticShapes import icosphere  # noqa: E402


def register(x0, F, x1, dtype, target=None, model=None, maxIter=1000, sigma=0.5, sigma_dist=0.3, time_step=0.1,
             scales=(1.0,), a0=None):
    K = Kernel(name='gauss', sigma=sigma)
    K.pk_dtype = dtype
    opts = dict(maxIter=maxIter, affine='none', regWeight=1.0, KparDiff=K, KparDist=('gauss', sigma_dist),
                sigmaError=1.0, errorType='varifold', pk_dtype=dtype, algorithm='bfgs', timeStep=time_step,
                verb=False, targetObjective=target, initialMomentum=a0)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    f = SecondOrderSurfaceMatching(Template=Surface(surf=(F, x0)), Target=Surface(surf=(F, x1)), options=opts)
    used = lp.warm_start(f, model, scales=scales) if model is not None else None
    f.optimizeMatching()
    torch.cuda.synchronize()
    return f, t0, time.perf_counter() - t0, used


def first_within(f, t0, target):
    for i, (e, t) in enumerate(zip(f.history, f.times)):
        if e <= target:
            return i + 1, t - t0
    return None, None


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--level', type=int, default=4)
    ap.add_argument('--pairs', type=int, default=20000)
    ap.add_argument('--heldout', type=int, default=2000)
    ap.add_argument('--eval', type=int, default=100)
    ap.add_argument('--epochs', type=int, default=8)
    ap.add_argument('--tol', type=float, default=1e-3)
    ap.add_argument('--seed', type=int, default=0)
    ap.add_argument('--scales', default='1.0;0.25,0.5,0.75,1.0',
                    help="learned variants separated by ';', each a comma-separated list of multiples of the proposal "
                         "tried at the start (the best one is kept)")
    ap.add_argument('--true-momentum', action='store_true',
                    help='also start BFGS from the momentum that generated the pair (the best a proposal could know)')
    ap.add_argument('--verbose', action='store_true')
    args = ap.parse_args()
    variants = [tuple(float(v) for v in grp.split(',')) for grp in args.scales.split(';')]
    x0, F = icosphere(args.level)
    t0 = time.perf_counter()
    feats, labels, momenta, n = lp.generate_pairs(x0, F, args.pairs, seed=args.seed)
    torch.cuda.synchronize()
    gen_s = time.perf_counter() - t0
    ntr = args.pairs - args.heldout
    model = lp.MomentumProposal(seed=args.seed)
    t0 = time.perf_counter()
    hist = lp.train(model, feats[:ntr], labels[:ntr], n, epochs=args.epochs, batch_pairs=16, lr=2e-3)
    torch.cuda.synchronize()
    train_s = time.perf_counter() - t0
    with torch.no_grad():
        ho = slice(ntr, ntr + min(args.heldout, 256))
        y = model.forward(feats[ho].reshape(-1, lp.IN_DIM)).reshape(-1, feats.shape[1], lp.OUT_DIM)[:, :n, :3]
        vel_err = float((y - labels[ho, :n]).norm() / labels[ho, :n].norm())
    del feats, labels
    torch.cuda.empty_cache()
    from base import pointEvolution as evol
    X0 = torch.from_numpy(x0).cuda()
    Kgen = Kernel(name='gauss', sigma=0.5)
    Kgen.pk_dtype = 'float64'
    rows = []
    for i in range(ntr, ntr + min(args.eval, args.heldout)):
        xt, _ = evol.shoot_second_order(X0, momenta[i], Kgen, 0.1)
        x1 = xt[-1].cpu().numpy()
        f64, t64, s64, _ = register(x0, F, x1, 'float64')
        estar = f64.history[-1]
        target = estar * (1 + args.tol)
        it64, s64_tol = first_within(f64, t64, target)
        f32, _, s32, _ = register(x0, F, x1, 'float32', target=target)
        row = {'pair': i, 'estar': estar, 'fp64_iters_to_tol': it64, 'fp64_s_to_tol': s64_tol,
               'fp64_iters_total': len(f64.history), 'fp32_iters': len(f32.history), 'fp32_s': s32,
               'fp32_reached': bool(f32.reached_target)}
        for v, scales in enumerate(variants):
            fl, _, sl, used = register(x0, F, x1, 'float32', target=target, model=model, scales=scales)
            row.update({f'learned{v}_iters': len(fl.history), f'learned{v}_s': sl,
                        f'learned{v}_reached': bool(fl.reached_target), f'learned{v}_used': used[0],
                        f'learned{v}_obj_ratio': used[1] / used[2], f'learned{v}_scale': used[3]})
        if args.true_momentum:
            ft, _, st_, _ = register(x0, F, x1, 'float32', target=target, a0=momenta[i].cpu().numpy())
            row.update({'true_iters': len(ft.history), 'true_s': st_, 'true_reached': bool(ft.reached_target)})
        rows.append(row)
        if args.verbose:
            print(json.dumps(row), flush=True)

    def stats(key):
        v = [r[key] for r in rows if r[key] is not None]
        return {'mean': statistics.fmean(v), 'median': statistics.median(v)} if v else None

    summary = {'experiment': 'learned proposal, held-out shot pairs', 'level': args.level, 'vertices': int(n),
               'pairs': args.pairs, 'trained_on': ntr, 'heldout': args.heldout, 'evaluated': len(rows),
               'epochs': args.epochs, 'generate_s': gen_s, 'train_s': train_s,
               'loss_first_last': [hist[0], hist[-1]], 'heldout_label_rel_err': vel_err, 'tol': args.tol,
               'fp64_plain_iters_to_tol': stats('fp64_iters_to_tol'), 'fp64_plain_s_to_tol': stats('fp64_s_to_tol'),
               'fp32_plain_iters': stats('fp32_iters'), 'fp32_plain_s': stats('fp32_s'),
               'fp32_plain_all_reached': all(r['fp32_reached'] for r in rows)}
    for v, scales in enumerate(variants):
        summary[f'learned{v}'] = {'scales': scales, 'iters': stats(f'learned{v}_iters'), 's': stats(f'learned{v}_s'),
                                  'used_frac': sum(r[f'learned{v}_used'] for r in rows) / max(len(rows), 1),
                                  'obj_proposal_over_zero': stats(f'learned{v}_obj_ratio'),
                                  'all_reached': all(r[f'learned{v}_reached'] for r in rows)}
    if args.true_momentum:
        summary['true_momentum_start'] = {'iters': stats('true_iters'), 's': stats('true_s'),
                                          'all_reached': all(r['true_reached'] for r in rows)}
    print(json.dumps(summary), flush=True)


if __name__ == '__main__':
    main()
