"""Time the reference py-lddmm itself end to end on the level-4 registration (its float64 numba path).

    python oracle/time_reference_level4.py --ref <the reference's py-lddmm directory> --order second --iters 50

Problem: icosphere level 4 (2,562 vertices) -> bumpy ellipsoid (8 bumps, amplitude 0.05, width 0.3, seed 0),
Gaussian deformation kernel sigma 0.5, unoriented varifold sigma 0.3, sigmaError 1, regWeight 1, T = 10, BFGS,
pk_dtype float64. Prints one JSON line with the wall time (JIT warm-up included and reported separately), the
iterations run and the objective history. Needs the reference tree (the shims of tests/golden/make_golden.py);
it is a measurement recipe for the CPU baseline (run by hand where the reference is present), not part of the
product, and nothing imports it.
"""
import argparse
import json
import logging
import os
import sys
import tempfile
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), 'tests', 'golden'))

import numpy as np  # noqa: E402

from make_golden import install_shims, load_shapes  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--ref', required=True, help='the py-lddmm directory of the reference tree')
    ap.add_argument('--order', default='second', choices=['first', 'second'])
    ap.add_argument('--iters', type=int, default=50)
    ap.add_argument('--level', type=int, default=4)
    args = ap.parse_args()
    logging.disable(logging.WARNING)
    install_shims()
    sys.path.insert(0, args.ref)
    sys.path.insert(0, os.path.join(args.ref, 'base'))
    from base import kernelFunctions as kf, surfaces as surf, surfaceDistances as sd
    sys.modules['base.surfaceDistancess'] = sd
    import base.pointset_distances as psd
    sys.modules['pointset_distances'] = psd
    from base import surfaceMatching as sm_mod, secondOrderSurfaceMatching as so_mod
    shapes = load_shapes()
    x0, F = shapes.icosphere(args.level)
    x1 = shapes.bumpy_ellipsoid(x0, seed=0)
    cls = so_mod.SecondOrderSurfaceMatching if args.order == 'second' else sm_mod.SurfaceMatching
    # JIT warm-up on a tiny problem (numba compiles each kernel once per process)
    xw, Fw = shapes.icosphere(1)
    t0 = time.perf_counter()
    with tempfile.TemporaryDirectory() as tmp:
        opts = dict(outputDir=tmp, mode='normal', maxIter=1, affine='none', regWeight=1.0,
                    KparDiff=kf.Kernel(name='gauss', sigma=0.5), KparDist=('gauss', 0.3), sigmaError=1.0,
                    errorType='varifold', pk_dtype='float64', algorithm='bfgs', timeStep=0.1, saveRate=10 ** 6,
                    verb=False)
        cls(Template=surf.Surface(surf=(Fw, xw)), Target=surf.Surface(surf=(Fw, shapes.bumpy_ellipsoid(xw))),
            options=opts).optimizeMatching()
    jit = time.perf_counter() - t0
    objs = []
    with tempfile.TemporaryDirectory() as tmp:
        opts = dict(outputDir=tmp, mode='normal', maxIter=args.iters, affine='none', regWeight=1.0,
                    KparDiff=kf.Kernel(name='gauss', sigma=0.5), KparDist=('gauss', 0.3), sigmaError=1.0,
                    errorType='varifold', pk_dtype='float64', algorithm='bfgs', timeStep=0.1, saveRate=10 ** 6,
                    verb=False)
        t0 = time.perf_counter()
        f = cls(Template=surf.Surface(surf=(F, x0)), Target=surf.Surface(surf=(F, x1)), options=opts)
        orig = f.endOfIteration

        def eoi(*a, **k):
            r = orig(*a, **k)
            objs.append(float(f.obj))
            return r
        f.endOfIteration = eoi
        f.optimizeMatching()
        wall = time.perf_counter() - t0
    print(json.dumps({'order': args.order, 'level': args.level, 'iters': len(objs), 'wall_s': wall, 'jit_s': jit,
                      'threads': int(os.environ.get('NUMBA_NUM_THREADS', os.cpu_count())), 'objs': objs}))


if __name__ == '__main__':
    main()
