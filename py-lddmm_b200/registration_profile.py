"""A few BFGS iterations of one registration, for a kernel launch list (which kernels a registration spends its
time in).

    python py-lddmm_b200/registration_profile.py [--level 6] [--iters 3] [--dtype float32]

Problem: the level-`--level` icosphere -> bumpy ellipsoid, SecondOrderSurfaceMatching with Gaussian sigma 0.5,
unoriented varifold sigma 0.2, sigmaError 1, T = 20, BFGS, from zero momentum. Prints the wall time per iteration.
"""
import argparse
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import torch  # noqa: E402

from base.kernelFunctions import Kernel  # noqa: E402
from base.surfaceMatching import SecondOrderSurfaceMatching  # noqa: E402
from base.surfaces import Surface  # noqa: E402
from base.syntheticShapes import icosphere, bumpy_ellipsoid  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--level', type=int, default=6)
    ap.add_argument('--iters', type=int, default=3)
    ap.add_argument('--dtype', default='float32', choices=['float32', 'float64'])
    args = ap.parse_args()
    x0, F = icosphere(args.level)
    x1 = bumpy_ellipsoid(x0, seed=0)
    K = Kernel(name='gauss', sigma=0.5)
    K.pk_dtype = args.dtype
    opts = dict(maxIter=args.iters, affine='none', regWeight=1.0, KparDiff=K, KparDist=('gauss', 0.2),
                sigmaError=1.0, errorType='varifold', pk_dtype=args.dtype, algorithm='bfgs', timeStep=0.05,
                verb=False)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    f = SecondOrderSurfaceMatching(Template=Surface(surf=(F, x0)), Target=Surface(surf=(F, x1)), options=opts)
    f.optimizeMatching()
    torch.cuda.synchronize()
    s = time.perf_counter() - t0
    print(json.dumps({'level': args.level, 'dtype': args.dtype, 'iters': args.iters, 's': s,
                      's_per_iter': s / args.iters, 'objective': f.history[-1]}))


if __name__ == '__main__':
    main()
