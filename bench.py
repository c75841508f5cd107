"""Benchmark of the B200 point-set hot path: Gaussian kernel pair-evaluations per second, plus the registration
half of the headline metric (seconds per registration pair to 1e-3 relative energy, learned vs plain).

Default run (the one-line JSON contract):
  workload  "L6 kernel sums": source vertices of the level-6 icosphere (N = M = 40,962), smoothed momenta
            a = K_0.3 (N(0, 0.1^2)), Gaussian widths sigma = 0.25 and 0.5. One step = K(x, x) a for both widths
            (2 N^2 pair evaluations), FP32 pair arithmetic with compensated accumulation and FP64 outputs.
  value     pairs/s with inputs resident in HBM, device-timed (CUDA events per step, L2 flushed between steps by
            writing a 256 MiB buffer; the flush is outside the timed events)
  e2e       the same step through the reference-facing API `Kernel.applyK(x, a)` with numpy (host) arrays:
            host->device copy of x and a, the kernels, device->host copy of the result, every step
  roofline  the pair kernel against the MUFU (ex2) pipe, its binding pipe: 1 SFU op + 6 FP32 lane-ops per pair
            (expanded-distance form); peak = 148 SMs x 16 MUFU lanes x max SM clock (the FP32 fraction beside it
            against 148 x 128 FP32 lanes); `traffic` = DRAM bytes per launch from the committed ncu capture of the
            same kernel, reported only while the kernel sources hash to the captured ones
  cpu_baseline  the CPU oracle (numba, float64, all host threads) on a bounded sample of the same sums; the
            oracle restates the reference's numba kernels without their per-pair temporaries, so it is faster
            than the reference's own `applyK_numba`, whose measured figure is carried beside it
  errors    relative error of the FP32 path against the FP64 GPU path (which matches the reference's goldens to
            1e-12) at level 6 with the level-6 registration's widths: the kernel sums, one second-order forward and
            one adjoint step, the varifold energy and gradient, and the registration objective and its gradient
  registration  (1 GPU) seconds per registration pair to reach (E - E*)/E* <= 1e-3 on the level-6 icosphere ->
            bumpy ellipsoid problem: E* is derived in the run by the plain FP64 path from zero momentum to the
            reference's BFGS stopping rule; the plain FP64 time to tolerance is read off the same run; then the
            plain FP32 path and the FP32 path from the learned warm start, each stopped at E* (1 + 1e-3; the
            warm-started registrations: median of 3 after one untimed run). The
            network is trained in the run on pairs the method generates (20,000 pairs: 18,000 trained on, 2,000
            held out), and a few held-out pairs are registered with and without it. Skipped with --no-registration.

Other modes (`--mode`, one JSON line per item, 1 GPU):
  ops                    per-operator device time and pipe fractions of the hot kernels at a level
  registration-profile   a few BFGS iterations of the level-6 registration (for a kernel launch list under ncu)
  large-registration     the level-7 registration (163,842 vertices, 32 bumps, sigma 0.3, varifold 0.1): E* from
                         the FP32 run to the stopping rule re-evaluated in FP64; the FP64 time to tolerance is an
                         estimate from its measured first iterations (labelled as such)
  proposal-eval          held-out evaluation of the learned proposal on level-4 shot pairs
  sharded-registration   (torchrun, N GPUs) one registration with its shooting / adjoint rows sharded over the
                         ranks (strong scaling), seconds per iteration as the max over ranks

`--impl reference` times the CPU implementation of the same sums (the oracle restatement of the reference's numba
kernels, all host threads) and prints the same metric with "impl": "reference".

Multi-GPU (torchrun): every rank runs the same workload on its own GPU (independent replicas, weak scaling); times
are the max over ranks; value = pairs of all ranks / that time.
"""
import argparse
import hashlib
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, 'py-lddmm_b200'))
sys.path.insert(0, REPO)

LEVEL = 6
SIGMAS = (0.25, 0.5)
# The self-sum K(x,x)a runs the symmetric expanded-distance kernel (pairs_kernel_symx<OpKSym, 128, 8>): rows in
# blocks of 128 x 8 points; an unordered pair of different blocks costs 9 FP32 lane-ops and one ex2 (row term,
# column term, the expanded squared distance), an ordered pair inside a block 6 and one ex2 (row term only).
KSYM_BLOCK = 1024
OPS_FP32_OFFDIAG, OPS_FP32_DIAG, OPS_SFU_PER_PAIR = 9, 6, 1
METRIC = 'Gauss kernel pairs/s'
# Coarse-to-fine warm start of the registrations: the coarse levels (icosphere levels of the source) per fine level,
# and the relative objective decrease over 3 iterations below which a coarse level hands over to the next. At level
# 6 one coarse level (4) measured faster than two (4, 5) on every seed tried: the level-5 stage costs more than the
# fine iteration it saves.
COARSE_LEVELS = {5: (3,), 6: (4,), 7: (4, 5)}
COARSE_RTOL = 1e-4


def coarse_templates(level, levels=None):
    """Coarser triangulations (faces, vertices) of the level-`level` icosphere source, coarsest first."""
    from base.syntheticShapes import icosphere
    levels = COARSE_LEVELS.get(level, ()) if levels is None else levels
    return [icosphere(lc)[::-1] for lc in levels if lc < level]
# The reference's own numba applyK (ku.applyK_numba, float64) at N = M = 40,962: 22.2 s per call on 8 threads of an
# Intel Xeon at 2.70 GHz, measured by importing the reference tree (which this benchmark does not read at run time).
REFERENCE_NUMBA_APPLYK = {'value': 7.56e7, 'unit': 'pairs/s', 'cores': 8,
                          'sample': 'one L6 applyK call (N=M=40,962, sigma 0.5), reference numba path, float64'}


def workload():
    from base.syntheticShapes import icosphere
    x, _ = icosphere(LEVEL)
    rng = np.random.default_rng(1)
    a_raw = rng.normal(0.0, 0.1, size=x.shape)
    return x, a_raw


def sym_pair_counts(n, block=KSYM_BLOCK):
    """(ordered pairs evaluated inside row blocks, unordered pairs evaluated between blocks) of one symmetric K(x,x)a."""
    nblk = (n + block - 1) // block
    sizes = [block] * (nblk - 1) + [n - block * (nblk - 1)]
    diag = sum(b * b for b in sizes)
    return diag, (n * n - diag) // 2


def config(n):
    return {'workload': 'L6 kernel sums: K(x,x)a, icosphere level 6, N=M=%d, sigma in %s, smoothed momenta' % (
        n, list(SIGMAS)), 'level': LEVEL, 'n_points': n, 'sigmas': list(SIGMAS), 'op': 'applyK (Gaussian)',
        'pairs_counted': 'N(N+1)/2 per sum: the symmetric kernel evaluates each unordered pair once and credits '
                         'both points (nm_equivalent_pairs_per_s counts the N*N ordered pairs of the same sums; '
                         'the CPU baseline and the reference arm evaluate and count all N*N)',
        'arithmetic': 'FP32 pair sums with compensated (two-sum) accumulation, FP64 outputs',
        'l2': 'flushed between timed steps (256 MiB write)'}


class ClockSampler:
    """nvidia-smi sampling (50 ms) of SM clock and throttle reasons; samples are kept for the timed window only
    (window = [mark_start, mark_end] wall clock, widened to the nearest samples when shorter than the period)."""

    NAMES = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None
        self.t0 = self.t1 = None
        # raw samples: $LDDMM_CLOCK_LOG (a directory) if set, else the system temporary directory
        base = os.environ.get('LDDMM_CLOCK_LOG') or tempfile.gettempdir()
        self.path = os.path.join(base, f'clocks_rank{device_index}.csv')

    def _gpu_id(self):
        try:
            import torch
            u = str(torch.cuda.get_device_properties(self.dev).uuid)
            return u if u.startswith('GPU-') else 'GPU-' + u
        except Exception:
            return str(self.dev)

    def __enter__(self):
        os.makedirs(os.path.dirname(self.path), exist_ok=True)
        q = ('timestamp,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,'
             'clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,'
             'clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap')
        try:
            self.fh = open(self.path, 'w')
            self.proc = subprocess.Popen(['nvidia-smi', '-i', self._gpu_id(), f'--query-gpu={q}',
                                          '--format=csv,noheader,nounits', '-lms', '50'], stdout=self.fh,
                                         stderr=subprocess.DEVNULL)
            deadline = time.time() + 5.0
            while time.time() < deadline and os.path.getsize(self.path) == 0:
                time.sleep(0.05)
        except Exception:
            self.proc = None
        return self

    def mark_start(self):
        self.t0 = time.time()

    def mark_end(self):
        self.t1 = time.time()
        time.sleep(0.12)

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.fh.close()

    def summary(self):
        import datetime
        rows = []
        try:
            for line in open(self.path):
                f = [t.strip() for t in line.split(',')]
                if len(f) < 9:
                    continue
                try:
                    ts = datetime.datetime.strptime(f[0], '%Y/%m/%d %H:%M:%S.%f').timestamp()
                    rows.append((ts, float(f[1]), float(f[2]), [v.lower() == 'active' for v in f[5:9]]))
                except ValueError:
                    continue
        except OSError:
            pass
        if not rows:
            return {'sm_mhz': None, 'sm_max_mhz': None, 'reasons': [], 'samples': 0}
        t0 = self.t0 if self.t0 is not None else rows[0][0]
        t1 = self.t1 if self.t1 is not None else rows[-1][0]
        sel = [r for r in rows if t0 - 0.06 <= r[0] <= t1 + 0.06]
        if not sel:   # window shorter than the sampling period: nearest sample after the start
            sel = [min(rows, key=lambda r: abs(r[0] - t0))]
        reasons = sorted({nm for r in sel for nm, on in zip(self.NAMES, r[3]) if on})
        return {'sm_mhz': statistics.median(r[1] for r in sel), 'sm_max_mhz': max(r[2] for r in sel),
                'reasons': reasons, 'samples': len(sel), 'window_s': round(t1 - t0, 4)}


def measured_peaks():
    p = os.path.join(REPO, 'MEASURED_PEAKS.json')
    try:
        return json.load(open(p))
    except Exception:
        return {}


def kernel_sources_sha16():
    """Hash of the CUDA sources that build the pair kernels (csrc/*.cu, *.cuh): ties an ncu capture to a kernel."""
    h = hashlib.sha256()
    csrc = os.path.join(REPO, 'py-lddmm_b200', 'csrc')
    for f in sorted(os.listdir(csrc)):
        if f.endswith(('.cu', '.cuh')):
            h.update(f.encode())
            h.update(open(os.path.join(csrc, f), 'rb').read())
    return h.hexdigest()[:16]


def ncu_traffic():
    """DRAM bytes per launch of the pair kernel from the committed ncu capture (profiles/applyk_pairs_L6_ncu.json),
    returned only when the capture was taken of the current kernel sources (their hash is stored with it)."""
    p = os.path.join(REPO, 'profiles', 'applyk_pairs_L6_ncu.json')
    try:
        d = json.load(open(p))
    except Exception:
        return None, 'no capture'
    if d.get('csrc_sha16') != kernel_sources_sha16():
        return None, 'capture of other kernel sources (stale): re-capture with the command in the json'
    return d.get('dram_bytes_per_launch'), f"ncu capture ({d.get('command', '')})"


def cpu_baseline(x, a, n_targets, threads, min_seconds=10.0, start=0):
    """Oracle (numba float64) on a bounded sample: blocks of n_targets targets x all sources x both widths, over
    successive target blocks from row `start`, until at least `min_seconds` have been measured (one block at least)."""
    import oracle as O
    O.apply_k(x[:64], x[:64], a[:64], SIGMAS[0])      # JIT warm-up
    pairs, dt = 0, 0.0
    start %= x.shape[0]
    while True:
        y = x[start:start + n_targets]
        t0 = time.perf_counter()
        for s in SIGMAS:
            O.apply_k(y, x, a, s)
        dt += time.perf_counter() - t0
        pairs += len(SIGMAS) * y.shape[0] * x.shape[0]
        start = (start + n_targets) % x.shape[0]
        if dt >= min_seconds:
            return pairs / dt, dt, pairs


def run_reference(args, rank, world):
    if rank != 0:
        return
    import numba
    threads = numba.config.NUMBA_NUM_THREADS       # every host thread numba may use (NUMBA_NUM_THREADS caps it)
    numba.set_num_threads(threads)
    x, a_raw = workload()
    import oracle as O
    t0 = time.perf_counter()
    a = O.apply_k(x, x, a_raw, 0.3)        # momentum smoothing (setup, untimed)
    setup = time.perf_counter() - t0
    n_t = args.ref_targets
    for _ in range(args.warmup):
        O.apply_k(x[:256], x, a, SIGMAS[0])
    vals = []
    for step in range(args.steps):
        v, dt, pairs = cpu_baseline(x, a, n_t, threads, min_seconds=0.0, start=step * n_t)
        vals.append((v, dt, pairs))
    tot_pairs = sum(p for _, _, p in vals)
    tot_t = sum(d for _, d, _ in vals)
    value = tot_pairs / tot_t
    line = {'metric': METRIC, 'value': value, 'unit': 'pairs/s', 'n_gpus': world, 'steps': args.steps,
            'warmup': args.warmup, 'ms_per_step': 1e3 * tot_t / args.steps, 'higher_is_better': True,
            'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f64', 'data': 'synthetic', 'impl': 'reference',
            'config': config(x.shape[0]),
            'cpu_baseline': {'value': value, 'unit': 'pairs/s', 'cores': threads, 'kind': 'port',
                             'sample': f'{n_t} targets x {x.shape[0]} sources x {len(SIGMAS)} widths per step '
                                       f'(port: the oracle numba restatement of ku.applyK_numba, float64, without '
                                       f'its per-pair temporaries)',
                             'reference_numba_applyK': REFERENCE_NUMBA_APPLYK},
            'e2e': {'value': value, 'unit': 'pairs/s', 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0},
            'setup_s': setup}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------------------------------------------
# Error statement of the FP32 path at level 6 (the level-6 registration's widths)
# ---------------------------------------------------------------------------------------------------------------
def _rel(a, b):
    import torch
    a, b = torch.as_tensor(a, dtype=torch.float64), torch.as_tensor(b, dtype=torch.float64)
    nb = float(b.norm())
    return float((a - b).norm()) / (nb if nb > 0 else 1.0)


def _step_increments(X, A, sigma, dt, precision):
    """(x1 - x)/dt and (a1 - a)/dt of one second-order forward step."""
    import torch
    from base import _native as nat
    n = X.shape[0]
    x1, a1 = torch.empty_like(X), torch.empty_like(X)
    ws, wsb = nat.workspace(n, n, precision)
    nat.check(nat.lib().lddmm_second_order_step(nat.ptr(X), nat.ptr(A), n, sigma, nat.KERNEL_GAUSS, dt,
                                                nat.origin_arg(nat.centroid(X)), nat.ptr(x1), nat.ptr(a1), precision,
                                                ws, wsb, nat.stream_ptr()), 'second_order_step')
    return (x1 - X) / dt, (a1 - A) / dt


def _adjoint_increments(X, A, PX, PA, sigma, dt, precision):
    import torch
    from base import _native as nat
    n = X.shape[0]
    p0, q0 = torch.empty_like(X), torch.empty_like(X)
    ws, wsb = nat.workspace(n, n, precision)
    nat.check(nat.lib().lddmm_second_order_adjoint_step(nat.ptr(X), nat.ptr(A), nat.ptr(PX), nat.ptr(PA), n, sigma,
                                                        nat.KERNEL_GAUSS, dt, nat.origin_arg(nat.centroid(X)),
                                                        nat.ptr(p0), nat.ptr(q0), precision, ws, wsb,
                                                        nat.stream_ptr()), 'second_order_adjoint_step')
    return (p0 - PX) / dt, (q0 - PA) / dt


def run_errors(level=6, sigmas=SIGMAS, sigma_dist=0.2, time_step=0.05):
    """Relative L2 error (relative difference for scalars) of the FP32 compensated path against the FP64 GPU path,
    which is pinned to the reference's own outputs at 1e-12. Inputs: the level-6 icosphere, momenta smoothed by K_0.3
    and scaled to an initial speed of 0.3 (as in the registrations), covectors px = minus the varifold gradient at
    a deformed surface and pa smoothed, the bumpy-ellipsoid target."""
    import torch
    from base import _native as nat
    from base.kernelFunctions import Kernel
    from base.surfaceDistances import SurfaceDataTerm
    from base.surfaceMatching import SecondOrderSurfaceMatching
    from base.surfaces import Surface
    from base.syntheticShapes import icosphere, bumpy_ellipsoid

    def K(s, dt):
        k = Kernel(name='gauss', sigma=s)
        k.pk_dtype = dt
        return k

    x, F = icosphere(level)
    x1 = bumpy_ellipsoid(x, seed=0)
    X = torch.from_numpy(x).cuda()
    rng = np.random.default_rng(7)
    K03 = K(0.3, 'float64')
    A = K03.applyK(X, torch.from_numpy(rng.normal(0, 0.1, x.shape)).cuda())
    A = A * (0.3 / K(0.5, 'float64').applyK(X, A).norm(dim=1).max())
    PA = K03.applyK(X, torch.from_numpy(rng.normal(0, 0.1, x.shape)).cuda())
    Xdef = X + 0.5 * K(0.5, 'float64').applyK(X, A)
    term = {p: SurfaceDataTerm(F, x1, F, K(sigma_dist, 'float64' if p == nat.FP64 else 'float32'), kind='varifold',
                               precision=p) for p in (nat.FP32C, nat.FP64)}
    PX = -term[nat.FP64].gradient(Xdef)
    out = {'reference': 'FP64 GPU path (pinned to the reference goldens at 1e-12)',
           'inputs': f'icosphere L{level} ({x.shape[0]} vertices, {F.shape[0]} faces); momenta K_0.3 N(0,0.1^2) at '
                     f'initial speed 0.3; px = -varifold gradient at a deformed surface; pa = K_0.3 N(0,0.1^2)',
           'metric': 'relative L2 error of each output array; relative difference of scalars'}
    for s in sigmas:
        k32, k64 = K(s, 'float32'), K(s, 'float64')
        e = {}
        e['applyK'] = _rel(k32.applyK(X, A), k64.applyK(X, A))
        e['applyDiffKT_lddmm'] = _rel(k32.applyDiffKT(X, PX, A, lddmm=True, regweight=1.0),
                                      k64.applyDiffKT(X, PX, A, lddmm=True, regweight=1.0))
        e['applyDDiffK11and12'] = _rel(k32.applyDDiffK11and12(X, A, A, PA), k64.applyDDiffK11and12(X, A, A, PA))
        e['applyDiffK1and2'] = _rel(k32.applyDiffK1and2(X, PA, A), k64.applyDiffK1and2(X, PA, A))
        sx32, sa32 = _step_increments(X, A, s, time_step, nat.FP32C)
        sx64, sa64 = _step_increments(X, A, s, time_step, nat.FP64)
        e['second_order_step'] = {'x_increment': _rel(sx32, sx64), 'a_increment': _rel(sa32, sa64)}
        bx32, ba32 = _adjoint_increments(X, A, PX, PA, s, time_step, nat.FP32C)
        bx64, ba64 = _adjoint_increments(X, A, PX, PA, s, time_step, nat.FP64)
        e['second_order_adjoint_step'] = {'px_increment': _rel(bx32, bx64), 'pa_increment': _rel(ba32, ba64)}
        # the registration objective 0.5 a0.K(x0)a0 + varifold(x_T, target) and its gradient, T = 20, at a0 = A
        obj, grad = {}, {}
        for dt in ('float32', 'float64'):
            opts = dict(maxIter=1, affine='none', regWeight=1.0, KparDiff=K(s, dt), KparDist=('gauss', sigma_dist),
                        sigmaError=1.0, errorType='varifold', pk_dtype=dt, algorithm='bfgs', timeStep=time_step,
                        verb=False, initialMomentum=A)
            f = SecondOrderSurfaceMatching(Template=Surface(surf=(F, x)), Target=Surface(surf=(F, x1)), options=opts)
            obj[dt] = f.objectiveFun()
            grad[dt] = f.getGradient(1.0)['a0']
        e['registration_objective'] = abs(obj['float32'] - obj['float64']) / abs(obj['float64'])
        e['registration_gradient'] = _rel(grad['float32'], grad['float64'])
        out[f'sigma_{s}'] = e
    e32 = term[nat.FP32C].energy(Xdef)[0]
    e64 = term[nat.FP64].energy(Xdef)[0]
    out[f'varifold_sigma_{sigma_dist}'] = {'energy': abs(float(e32) - float(e64)) / abs(float(e64)),
                                           'gradient': _rel(term[nat.FP32C].gradient(Xdef), -PX)}
    return out


# ---------------------------------------------------------------------------------------------------------------
# Registration: seconds per pair to 1e-3 relative energy
# ---------------------------------------------------------------------------------------------------------------
def _matching(x0, F, x1, dtype, sigma, sigma_dist, time_step, target=None, maxIter=600, a0=None):
    from base.kernelFunctions import Kernel
    from base.surfaceMatching import SecondOrderSurfaceMatching
    from base.surfaces import Surface
    K = Kernel(name='gauss', sigma=sigma)
    K.pk_dtype = dtype
    opts = dict(maxIter=maxIter, affine='none', regWeight=1.0, KparDiff=K, KparDist=('gauss', sigma_dist),
                sigmaError=1.0, errorType='varifold', pk_dtype=dtype, algorithm='bfgs', timeStep=time_step, verb=False,
                targetObjective=target, initialMomentum=a0)
    return SecondOrderSurfaceMatching(Template=Surface(surf=(F, x0)), Target=Surface(surf=(F, x1)), options=opts)


def _register(x0, F, x1, dtype, sigma, sigma_dist, time_step, target=None, model=None, scales=(0.5, 0.75, 1.0),
              maxIter=600, a0=None, coarse=None, coarse_rtol=COARSE_RTOL):
    """One registration, timed from construction to the end (device synchronised): (matching, t0, seconds,
    warm-start record). With `target`, BFGS stops at the end of the first iteration at or below it. With `coarse`
    (coarser triangulations (faces, vertices) of the source, coarsest first) the warm start is the coarse-to-fine one
    (learnedProposal.multilevel_warm_start, with the network at the coarsest level when `model` is given);
    otherwise the network's proposal at this level (learnedProposal.warm_start) when `model` is given."""
    import gc
    import torch
    from base import learnedProposal as lp
    gc.collect()            # not inside the timed region: a cyclic-GC pass there would land on one run at random
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    f = _matching(x0, F, x1, dtype, sigma, sigma_dist, time_step, target=target, maxIter=maxIter, a0=a0)
    if coarse is not None:
        used = lp.multilevel_warm_start(f, model, coarse, rtol=coarse_rtol, scales=scales)
    else:
        used = lp.warm_start(f, model, scales=scales) if model is not None else None
    f.optimizeMatching()
    torch.cuda.synchronize()
    return f, t0, time.perf_counter() - t0, used


# The warm-started registrations take a fraction of a second, within reach of host-side jitter (their coarse levels
# are launch-bound): each is timed WARM_REPEATS times after one untimed run of the same path, and the median kept.
WARM_REPEATS = 3


def _register_median(*a, repeats=WARM_REPEATS, **k):
    """_register `repeats` times: (matching and record of the median run, median seconds, every sample). The caching
    allocator keeps its blocks between the repeats (no cudaMalloc inside the timed region after the first)."""
    runs = []
    for _ in range(repeats):
        f, _, t, used = _register(*a, **k)
        runs.append((t, f, used))
    runs.sort(key=lambda r: r[0])
    t, f, used = runs[len(runs) // 2]
    return f, t, [r[0] for r in runs], used


def _first_within(f, t0, target):
    """Iterations and seconds (from t0) to the first BFGS iterate at or below target."""
    for i, (e, t) in enumerate(zip(f.history, f.times)):
        if e <= target:
            return i + 1, t - t0
    return None, None


def _fp64_energy(f):
    f.resetPK('float64')
    f.obj = None
    return float(f.objectiveFun())


def train_proposal(pairs, heldout, epochs, seed=0, law='shapes'):
    """Network trained on pairs the method generates at level 4 (the last `heldout` pairs never trained on);
    `law`: the momentum law of the generated pairs (learnedProposal.generate_pairs)."""
    import torch
    from base import learnedProposal as lp
    from base.syntheticShapes import icosphere
    xs, Fs = icosphere(4)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    feats, labels, momenta, n4 = lp.generate_pairs(xs, Fs, pairs, seed=seed, timeStep=0.1, law=law)
    torch.cuda.synchronize()
    t_gen = time.perf_counter() - t0
    model = lp.MomentumProposal(seed=seed)
    ntr = pairs - heldout
    t0 = time.perf_counter()
    hist = lp.train(model, feats[:ntr], labels[:ntr], n4, epochs=epochs, batch_pairs=16, lr=2e-3)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t0
    with torch.no_grad():
        ho = slice(ntr, ntr + min(heldout, 256))
        y = model.forward(feats[ho].reshape(-1, lp.IN_DIM)).reshape(-1, feats.shape[1], lp.OUT_DIM)[:, :n4, :3]
        err = float((y - labels[ho, :n4]).norm() / labels[ho, :n4].norm())
    rec = {'level': 4, 'pairs': pairs, 'train_pairs': ntr, 'heldout_pairs': heldout, 'epochs': epochs,
           'generate_s': t_gen, 'train_s': t_train, 'loss_first_last': [hist[0], hist[-1]],
           'heldout_label_rel_err': err,
           'momentum_law': lp.MOMENTUM_LAW if law == 'noise' else lp.MOMENTUM_LAW_SHAPES}
    del feats, labels
    torch.cuda.empty_cache()
    return model, rec, (xs, Fs, momenta[ntr:])


def heldout_registrations(model, heldset, count, tol=1e-3):
    """Registers `count` held-out shot pairs (level 4, sigma 0.5, varifold 0.3, T = 10): E* by plain FP64 to the
    stopping rule, then plain FP32 and learned FP32 to E* (1 + tol). Returns per-pair iterations and seconds."""
    import torch
    from base import pointEvolution as evol
    from base.kernelFunctions import Kernel
    xs, Fs, momenta = heldset
    X0 = torch.from_numpy(xs).cuda()
    Kg = Kernel(name='gauss', sigma=0.5)
    Kg.pk_dtype = 'float64'
    rows = []
    for i in range(min(count, momenta.shape[0])):
        xt, _ = evol.shoot_second_order(X0, momenta[i], Kg, 0.1)
        x1 = xt[-1].cpu().numpy()
        f64, t64, _, _ = _register(xs, Fs, x1, 'float64', 0.5, 0.3, 0.1)
        estar = f64.history[-1]
        target = estar * (1 + tol)
        it64, s64 = _first_within(f64, t64, target)
        f32, _, s32, _ = _register(xs, Fs, x1, 'float32', 0.5, 0.3, 0.1, target=target)
        fl, _, sl, used = _register(xs, Fs, x1, 'float32', 0.5, 0.3, 0.1, target=target, model=model)
        rows.append({'fp64_iters': it64, 'fp64_s': s64, 'fp32_iters': len(f32.history), 'fp32_s': s32,
                     'learned_iters': len(fl.history), 'learned_s': sl, 'proposal_used': used[0],
                     'reached': bool(f32.reached_target and fl.reached_target)})
    mean = lambda k: statistics.fmean(r[k] for r in rows if r[k] is not None)   # noqa: E731
    return {'pairs': len(rows), 'problem': 'level-4 held-out shot pairs, sigma 0.5, varifold 0.3, T=10',
            'plain_fp64_iters': mean('fp64_iters'), 'plain_fp32_iters': mean('fp32_iters'),
            'learned_fp32_iters': mean('learned_iters'), 'plain_fp64_s': mean('fp64_s'),
            'plain_fp32_s': mean('fp32_s'), 'learned_fp32_s': mean('learned_s'),
            'proposal_used_frac': sum(r['proposal_used'] for r in rows) / max(len(rows), 1),
            'all_reached': all(r['reached'] for r in rows)}


def heldout_ellipsoids(model, seeds, level, coarse, tol=1e-3):
    """Registrations of bumpy ellipsoids of other seeds (never the headline problem's seed 0), level `level`, sigma 0.5
    / varifold 0.2, T = 20: E* and the plain FP64 time to tolerance from the FP64 run to the stopping rule, then the
    plain FP32 path and the learned coarse-to-fine warm start to E* (1 + tol)."""
    import torch
    from base.syntheticShapes import icosphere, bumpy_ellipsoid
    x0, F = icosphere(level)
    rows = []
    for seed in seeds:
        x1 = bumpy_ellipsoid(x0, seed=seed)
        f64, t0, _, _ = _register(x0, F, x1, 'float64', 0.5, 0.2, 0.05)
        estar = f64.history[-1]
        target = estar * (1 + tol)
        it64, s64 = _first_within(f64, t0, target)
        del f64
        f32, _, s32, _ = _register(x0, F, x1, 'float32', 0.5, 0.2, 0.05, target=target)
        fl, sl, samples, rec = _register_median(x0, F, x1, 'float32', 0.5, 0.2, 0.05, target=target, model=model,
                                                coarse=coarse)
        rows.append({'seed': seed, 'estar': estar, 'plain_fp64_iters': it64, 'plain_fp64_s': s64,
                     'plain_fp32_iters': len(f32.history), 'plain_fp32_s': s32, 'learned_multilevel_fine_iters':
                     len(fl.history), 'learned_multilevel_s': sl, 'learned_multilevel_samples_s': samples,
                     'reached': bool(f32.reached_target and
                                                                                fl.reached_target),
                     'coarse_iters': [lv['iters'] for lv in rec['levels']], 'speedup_learned_vs_plain_fp64':
                     s64 / sl if s64 else None})
        del f32, fl
        torch.cuda.empty_cache()
    sp = [r['speedup_learned_vs_plain_fp64'] for r in rows if r['speedup_learned_vs_plain_fp64']]
    return {'problem': f'icosphere L{level} -> bumpy ellipsoids (8 bumps) of seeds {list(seeds)}, sigma 0.5 / '
                       'varifold 0.2, T=20', 'pairs': rows,
            'speedup_min': min(sp) if sp else None, 'speedup_geomean': float(np.exp(np.mean(np.log(sp)))) if sp
            else None}


def _levels_arg(args):
    v = getattr(args, 'coarse_levels', None)
    return None if v in (None, '') else tuple(int(t) for t in v.split(',') if t.strip())


def run_registration(args):
    """Seconds per registration pair to reach (E - E*)/E* <= 1e-3 on the level-6 icosphere -> bumpy ellipsoid problem
    (Gaussian sigma 0.5, varifold sigma 0.2, T = 20, sigmaError 1, BFGS): the plain FP64 path, the plain FP32 path,
    the FP32 path from the network's proposal at level 6, the FP32 path from the coarse-to-fine warm start without
    the network, and the learned warm start proper (network proposal at the coarsest level, plain BFGS at the
    coarse levels, prolongation; network trained here at level 4 on pairs generated by shooting)."""
    import torch
    from base.syntheticShapes import icosphere, bumpy_ellipsoid
    level, tol = args.reg_level, 1e-3
    x0, F = icosphere(level)
    x1 = bumpy_ellipsoid(x0, seed=0)
    sig, sigd, ts = 0.5, 0.2, 0.05
    levels = [lc for lc in (_levels_arg(args) or COARSE_LEVELS.get(level, ())) if lc < level]
    coarse = coarse_templates(level, levels)
    res = {'problem': f'icosphere L{level} ({x0.shape[0]} vertices) -> bumpy ellipsoid (8 bumps), sigma {sig} / '
                      f'varifold {sigd}, T={int(round(1 / ts))}, sigmaError 1, BFGS', 'criterion': '(E - E*)/E* <= 1e-3',
           'warm_start': {'coarse_levels': levels, 'coarse_rtol': COARSE_RTOL,
                          'coarse_stop': 'relative objective decrease over 3 iterations below coarse_rtol',
                          'prolongation': 'momentum density interpolated by a normalised Gaussian of 0.4 x the '
                                          'coarse mean edge length'}}
    # E*: the plain FP64 path run to the reference's stopping rule (|obj - obj_old| < 1e-7 after burn-in); its time
    # to tolerance is that of the same run's first iterate within tolerance
    f64, t0_64, s64_total, _ = _register(x0, F, x1, 'float64', sig, sigd, ts, maxIter=args.estar_iters)
    estar = f64.history[-1]
    target = estar * (1 + tol)
    it64, s64 = _first_within(f64, t0_64, target)
    res['estar'] = estar
    res['estar_run'] = {'iters': len(f64.history), 's': s64_total, 'converged': bool(f64.converged),
                        'stopping_rule': 'BFGS |obj - obj_old| < 1e-7 after burn-in, or gradient below threshold'}
    res['plain_fp64'] = {'s_per_pair': s64, 'iters': it64, 'reached': it64 is not None,
                         'rel_energy_fp64': (f64.history[it64 - 1] - estar) / abs(estar) if it64 else None,
                         'timed': 'same run as E*, to its first iterate within tolerance'}
    del f64
    torch.cuda.empty_cache()
    model, res['proposal'], heldset = train_proposal(args.train_pairs, args.heldout_pairs, args.train_epochs,
                                                     law=args.momentum_law)
    runs = (('plain_fp32', None, None), ('learned_fp32', model, None), ('multilevel_plain_fp32', None, coarse),
            ('learned_multilevel_fp32', model, coarse))
    # untimed: the first run of the coarse-to-fine path (its level-4 plans and workspaces, the prolongation's masses)
    _register(x0, F, x1, 'float32', sig, sigd, ts, target=target, model=model, coarse=coarse)
    for name, model_, coarse_ in runs:
        if coarse_ is None:
            f, t0, t, used = _register(x0, F, x1, 'float32', sig, sigd, ts, target=target, model=model_)
            samples = [t]
        else:
            f, t, samples, used = _register_median(x0, F, x1, 'float32', sig, sigd, ts, target=target, model=model_,
                                                   coarse=coarse_)
        e = _fp64_energy(f)
        res[name] = {'s_per_pair': t, 'iters': len(f.history), 'reached': bool(f.reached_target),
                     'rel_energy_fp64': (e - estar) / abs(estar)}
        if coarse_ is not None:
            res[name]['samples_s'] = samples
            res[name]['first_step_gap'] = used.get('first_step_gap')
            res[name].update({'fine_iters': len(f.history), 'coarse_iters': [lv['iters'] for lv in used['levels']],
                              'network_proposal_used': used['network_proposal_used'],
                              'prolonged_used': used['prolonged_used'],
                              'rel_obj_prolonged': (used['obj_prolonged'] - estar) / abs(estar)})
        elif used is not None:
            res[name].update({'proposal_used': used[0], 'obj_proposal': used[1], 'obj_zero': used[2],
                              'scale': used[3]})
        del f
    p64 = res['plain_fp64']['s_per_pair']
    res['speedup_learned_vs_plain_fp64'] = p64 / res['learned_multilevel_fp32']['s_per_pair']
    res['speedup_learned_single_level_vs_plain_fp64'] = p64 / res['learned_fp32']['s_per_pair']
    res['speedup_multilevel_plain_vs_plain_fp64'] = p64 / res['multilevel_plain_fp32']['s_per_pair']
    res['speedup_plain_fp32_vs_plain_fp64'] = p64 / res['plain_fp32']['s_per_pair']
    res['heldout'] = heldout_registrations(model, heldset, args.heldout_eval)
    seeds = [int(v) for v in args.heldout_seeds.split(',') if v.strip()] if args.heldout_seeds else []
    if seeds:
        res['heldout_ellipsoids'] = heldout_ellipsoids(model, seeds, level, coarse, tol)
    res['level4_fp64_50it'] = run_level4_fp64()
    return res


def run_level4_fp64():
    """The small CPU-runnable registration end to end: level-4 icosphere -> bumpy ellipsoid, sigma 0.5, varifold 0.3,
    sigmaError 1, T = 10, BFGS, 50 iterations, float64 (the FP64 path, both matching classes)."""
    import torch
    from base.kernelFunctions import Kernel
    from base.surfaceMatching import SurfaceMatching, SecondOrderSurfaceMatching
    from base.surfaces import Surface
    from base.syntheticShapes import icosphere, bumpy_ellipsoid
    x0, F = icosphere(4)
    x1 = bumpy_ellipsoid(x0, seed=0)
    out = {}
    for name, cls in (('second_order', SecondOrderSurfaceMatching), ('first_order', SurfaceMatching)):
        K = Kernel(name='gauss', sigma=0.5)
        K.pk_dtype = 'float64'
        opts = dict(maxIter=50, affine='none', regWeight=1.0, KparDiff=K, KparDist=('gauss', 0.3), sigmaError=1.0,
                    errorType='varifold', pk_dtype='float64', algorithm='bfgs', timeStep=0.1, verb=False)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        f = cls(Template=Surface(surf=(F, x0)), Target=Surface(surf=(F, x1)), options=opts)
        f.optimizeMatching()
        torch.cuda.synchronize()
        out[name] = {'s': time.perf_counter() - t0, 'iters': len(f.history), 'final_obj': f.history[-1]}
    return out


# ---------------------------------------------------------------------------------------------------------------
# Other modes
# ---------------------------------------------------------------------------------------------------------------
# FP32 lane-ops and SFU ops per pair of each kernel (packed instructions counted per lane); applyK, the second-order
# step and the varifold energy and gradient: their expanded-distance form (blocks whose radius is too large for it
# take the difference form: 9, 16, 12 and 22)
OP_COUNTS = {'applyK': (6, 1), 'applyDiffKT_lddmm': (16, 1), 'applyDDiffK11and12': (23, 1), 'applyDiffK1and2': (16, 1),
             'so_step': (14, 1), 'so_adjoint_step': (37, 1), 'fo_adjoint_step': (19, 1), 'varifold_energy': (9, 1),
             'varifold_gradient': (19, 1)}
# Self-sums that run a symmetric kernel (FP32, Gaussian): (row block size, FP32 lane-ops per ordered pair inside a
# block (row terms only), FP32 lane-ops per unordered pair between blocks (row and column terms)); one ex2 each.
SYM_COUNTS = {'applyK': (1024, 6, 9), 'so_step': (1024, 16, 22), 'so_adjoint_step': (512, 42, 51),
              'fo_adjoint_step': (512, 19, 25)}


def mode_ops(args):
    """Per-operator device time (CUDA events on the launching stream, after warm-up), pairs/s and FP32 / SFU pipe
    fractions (nominal pipe peaks at $SM_MHZ, default 1965). One JSON line per operator. With --reps 1 --warmup 0 it
    makes one launch per operator, for ncu captures."""
    import torch
    from base import _native as nat
    from base.surfaceDistances import vertex_face_table
    from base.syntheticShapes import icosphere, bumpy_ellipsoid
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

    XT = torch.stack([X, X])
    AT = A.unsqueeze(0).contiguous()
    PXT = torch.empty_like(XT)
    calls = {
        'applyK': lambda: ok(lib.lddmm_apply_k(p(X), n, p(X), p(A), n, s, kern, o, p(o1), prec, ws, wsb, st)),
        'applyDiffKT_lddmm': lambda: ok(lib.lddmm_apply_diff_kt(p(X), n, p(X), p(P), p(A), n, s, kern, 2, 1.0, o,
                                                                p(o1), prec, ws, wsb, st)),
        'applyDDiffK11and12': lambda: ok(lib.lddmm_apply_ddiff_k11and12(p(X), p(A), p(A), p(Q), n, s, kern, o, p(o1),
                                                                        prec, ws, wsb, st)),
        'applyDiffK1and2': lambda: ok(lib.lddmm_apply_diff_k1and2(p(X), p(Q), p(A), n, s, kern, o, p(o1), prec, ws,
                                                                  wsb, st)),
        'so_step': lambda: ok(lib.lddmm_second_order_step(p(X), p(A), n, s, kern, 0.05, o, p(o1), p(o2), prec, ws,
                                                          wsb, st)),
        'so_adjoint_step': lambda: ok(lib.lddmm_second_order_adjoint_step(p(X), p(A), p(P), p(Q), n, s, kern, 0.05,
                                                                          o, p(o1), p(o2), prec, ws, wsb, st)),
        'varifold_energy': lambda: ok(lib.lddmm_surface_energy(0, p(X), n, p(FF), nf, None, p(X1), n, p(FF), nf, None,
                                                               sd, o, 0, p(E), prec, sws, swsb, st)),
        'varifold_gradient': lambda: ok(lib.lddmm_surface_gradient(0, p(X), n, p(FF), nf, None, p(off), p(items),
                                                                   p(X1), n, p(FF), nf, None, sd, o, p(o1), None,
                                                                   prec, sws, swsb, st)),
        # the first-order adjoint entry point runs T steps: one step with a 2-state trajectory
        'fo_adjoint_step': lambda: ok(lib.lddmm_first_order_gradient(p(XT), p(AT), n, 1, s, kern, 1.0, p(P), 1, o,
                                                                     p(PXT), p(dat), prec, ws, wsb, st)),
    }
    pairs = {k: float(n) * n for k in calls}
    pairs['varifold_energy'] = pairs['varifold_gradient'] = float(nf) * 2 * nf
    props = torch.cuda.get_device_properties(0)
    sm_clock = float(os.environ.get('SM_MHZ', '1965'))
    peak32 = props.multi_processor_count * 128 * sm_clock * 1e6
    peaksfu = props.multi_processor_count * 16 * sm_clock * 1e6
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
        fp32, sfu = OP_COUNTS[name]
        gauss = kern == nat.KERNEL_GAUSS or name.startswith('varifold')   # the op counts are the Gaussian ones
        rec = {'op': name, 'kernel': args.kernel if not name.startswith('varifold') else 'gauss', 'level': args.level,
               'precision': args.precision, 'ms': round(ms, 4), 'pairs_per_s': pps,
               'frac_fp32_peak': pps * fp32 / peak32 if args.precision == 'fp32' and gauss else None,
               'frac_sfu_peak': pps * sfu / peaksfu if gauss else None}
        if name in SYM_COUNTS and args.precision == 'fp32' and kern == nat.KERNEL_GAUSS:
            blk, c_in, c_between = SYM_COUNTS[name]
            diag, between = sym_pair_counts(n, blk)
            rec.update({'kernel_form': 'symmetric', 'pairs_per_s': (diag + between) / (ms * 1e-3),
                        'nm_equivalent_pairs_per_s': pps,
                        'frac_fp32_peak': (c_in * diag + c_between * between) / (ms * 1e-3) / peak32,
                        'frac_sfu_peak': (diag + between) / (ms * 1e-3) / peaksfu})
        print(json.dumps(rec), flush=True)


def mode_registration_profile(args):
    """A few BFGS iterations of the level-6 registration (FP32 or FP64): wall time per iteration. With --warm
    multilevel, the coarse-to-fine warm start (without the network) runs first and the fine level then makes --iters
    iterations: the launch list of the registration path that the learned warm start takes."""
    from base.syntheticShapes import icosphere, bumpy_ellipsoid
    x0, F = icosphere(args.reg_level)
    x1 = bumpy_ellipsoid(x0, seed=0)
    dtype = 'float64' if args.precision == 'fp64' else 'float32'
    coarse = None
    if args.warm == 'multilevel':
        levels = [lc for lc in (_levels_arg(args) or COARSE_LEVELS.get(args.reg_level, ())) if lc < args.reg_level]
        coarse = coarse_templates(args.reg_level, levels)
    f, _, s, rec = _register(x0, F, x1, dtype, 0.5, 0.2, 0.05, maxIter=args.iters, coarse=coarse)
    out = {'level': args.reg_level, 'dtype': dtype, 'iters': args.iters, 's': s, 's_per_iter': s / args.iters,
           'objective': f.history[-1]}
    if coarse is not None:
        out['warm_start'] = {'coarse_iters': [lv['iters'] for lv in rec['levels']], 'prolonged_used':
                             rec['prolonged_used']}
    print(json.dumps(out), flush=True)


def mode_large_registration(args):
    """Level-7 registration (163,842 vertices, 327,680 faces, 32 bumps; sigma 0.3, varifold 0.1, T = 20):
      1. plain FP32 from zero momentum to the BFGS stopping rule; its final momentum re-evaluated on the FP64 path
         gives E*, and its first iterate within tolerance gives the plain FP32 iterations and seconds (the FP64 run
         to the stopping rule takes ~6 minutes; with --l7-fp64-full it is run too, and E*, its time to tolerance and
         the speed-ups are also reported from it, labelled measured);
      2. FP32 from the learned proposal (network trained at level 4, applied per vertex) to E* (1 + tol), and from
         the coarse-to-fine warm start with and without the network (coarse levels 4 and 5 by default);
      3. the plain FP64 path timed over --fp64-probe-iters iterations; its time to tolerance is ESTIMATED as its
         first iteration plus (plain FP32 iterations to tolerance - 1) x its later seconds per iteration."""
    import torch
    from base import learnedProposal as lp
    from base.syntheticShapes import icosphere, bumpy_ellipsoid
    tol, sig, sigd, ts = 1e-3, 0.3, 0.1, 0.05
    x0, F = icosphere(7)
    x1 = bumpy_ellipsoid(x0, n_bumps=32, seed=0)
    out = {'problem': f'icosphere L7 ({x0.shape[0]} vertices, {F.shape[0]} faces) -> bumpy ellipsoid (32 bumps), '
                      f'sigma {sig} / varifold {sigd}, T=20, sigmaError 1, BFGS', 'tol': tol}
    f32, t0, s32_total, _ = _register(x0, F, x1, 'float32', sig, sigd, ts, maxIter=args.estar_iters)
    estar = _fp64_energy(f32)
    target = estar * (1 + tol)
    it32, s32 = _first_within(f32, t0, target)
    out['plain_fp32'] = {'iters_total': len(f32.history), 'converged': bool(f32.converged), 's_total': s32_total,
                         'estar_fp64_of_fp32_optimum': estar, 'iters_to_tol': it32, 's_to_tol': s32}
    del f32
    torch.cuda.empty_cache()
    model, out['proposal'], _ = train_proposal(args.train_pairs, args.heldout_pairs, args.train_epochs,
                                               law=args.momentum_law)
    fl, _, sl, used = _register(x0, F, x1, 'float32', sig, sigd, ts, target=target, model=model)
    out['learned_fp32'] = {'iters': len(fl.history), 's_to_tol': sl, 'reached': bool(fl.reached_target),
                           'rel_energy_fp64': (_fp64_energy(fl) - estar) / abs(estar), 'proposal_used': used[0],
                           'obj_proposal': used[1], 'obj_zero': used[2], 'scale': used[3]}
    del fl
    torch.cuda.empty_cache()
    levels = [lc for lc in (_levels_arg(args) or COARSE_LEVELS.get(7, ())) if lc < 7]
    for name, model_ in (('multilevel_plain_fp32', None), ('learned_multilevel_fp32', model)):
        fm, _, sm_, rec = _register(x0, F, x1, 'float32', sig, sigd, ts, target=target, model=model_,
                                    coarse=coarse_templates(7, levels))
        out[name] = {'fine_iters': len(fm.history), 's_to_tol': sm_, 'reached': bool(fm.reached_target),
                     'rel_energy_fp64': (_fp64_energy(fm) - estar) / abs(estar), 'coarse_levels': levels,
                     'coarse_iters': [lv['iters'] for lv in rec['levels']],
                     'network_proposal_used': rec['network_proposal_used'], 'prolonged_used': rec['prolonged_used']}
        del fm
        torch.cuda.empty_cache()
    if args.l7_fp64_full:
        # the plain FP64 path run to the stopping rule: E* from FP64 itself and its measured time to tolerance
        f64, t0, s64_total, _ = _register(x0, F, x1, 'float64', sig, sigd, ts, maxIter=args.estar_iters)
        estar64 = f64.history[-1]
        it64, s64 = _first_within(f64, t0, estar64 * (1 + tol))
        out['plain_fp64_full'] = {'estar': estar64, 'iters_total': len(f64.history), 'converged': bool(f64.converged),
                                  's_total': s64_total, 'iters_to_tol': it64, 's_to_tol': s64,
                                  'estar_fp32_run_rel_diff': (estar - estar64) / abs(estar64)}
        for name in ('learned_multilevel_fp32', 'multilevel_plain_fp32', 'learned_fp32'):
            r = out[name]
            r['rel_energy_vs_fp64_estar'] = (estar * (1 + r['rel_energy_fp64']) - estar64) / abs(estar64)
        if s64 is not None:
            out['speedup_learned_vs_plain_fp64_measured'] = s64 / out['learned_multilevel_fp32']['s_to_tol']
            out['speedup_multilevel_plain_vs_plain_fp64_measured'] = s64 / out['multilevel_plain_fp32']['s_to_tol']
            out['speedup_plain_fp32_vs_plain_fp64_measured'] = s64 / s32 if s32 else None
        del f64
        torch.cuda.empty_cache()
    k = max(2, args.fp64_probe_iters)
    f64, t0, s64, _ = _register(x0, F, x1, 'float64', sig, sigd, ts, maxIter=k)
    first = f64.times[0] - t0
    per_it = (f64.times[k - 1] - f64.times[0]) / (k - 1)
    out['plain_fp64_probe'] = {'iters': k, 's': s64, 's_first_iter': first, 's_per_iter': per_it}
    if it32 is not None:
        est = first + per_it * (it32 - 1)
        out['plain_fp64_s_to_tol_ESTIMATE'] = est
        out['speedup_learned_vs_plain_fp64_ESTIMATE'] = est / out['learned_multilevel_fp32']['s_to_tol']
        out['speedup_learned_single_level_vs_plain_fp64_ESTIMATE'] = est / sl
        out['speedup_multilevel_plain_vs_plain_fp64_ESTIMATE'] = est / out['multilevel_plain_fp32']['s_to_tol']
        out['speedup_plain_fp32_vs_plain_fp64_ESTIMATE'] = est / s32
    print(json.dumps(out), flush=True)


def mode_sharded_registration(args, rank, world, local_rank):
    """One registration with its shooting and adjoint rows sharded over the torchrun ranks (strong scaling: the
    target rows of every step split over the ranks, one all-gather per step): the level-`--reg-level` problem (sigma 0.5, varifold 0.2, T = 20), FP32, `--iters` BFGS
    iterations from zero momentum; seconds per iteration as the max over ranks of each rank's device-synchronised
    wall time. Every rank ends with the same objective (checked)."""
    import datetime
    import torch
    import torch.distributed as dist
    from base.syntheticShapes import icosphere, bumpy_ellipsoid
    torch.cuda.set_device(local_rank)
    if world > 1:
        dist.init_process_group('nccl', timeout=datetime.timedelta(seconds=300))
    else:
        os.environ.setdefault('MASTER_ADDR', '127.0.0.1')
        os.environ.setdefault('MASTER_PORT', '29531')
        dist.init_process_group('nccl', rank=0, world_size=1)
    try:
        x0, F = icosphere(args.reg_level)
        x1 = bumpy_ellipsoid(x0, seed=0)
        f = _matching(x0, F, x1, 'float32', 0.5, 0.2, 0.05, maxIter=args.iters)
        f.options['processGroup'] = True
        f.objectiveFun()                     # warm-up: plans, workspaces, NCCL communicator
        f.obj = None
        torch.cuda.synchronize()
        dist.barrier()
        t0 = time.perf_counter()
        f.optimizeMatching()
        torch.cuda.synchronize()
        s = torch.tensor([time.perf_counter() - t0, f.history[-1]], dtype=torch.float64, device='cuda')
        smax = s.clone()
        dist.all_reduce(smax, op=dist.ReduceOp.MAX)
        smin = s.clone()
        dist.all_reduce(smin, op=dist.ReduceOp.MIN)
        if rank == 0:
            print(json.dumps({'mode': 'sharded-registration', 'n_gpus': world, 'level': args.reg_level,
                              'vertices': int(x0.shape[0]), 'iters': len(f.history), 's': float(smax[0]),
                              's_per_iter': float(smax[0]) / max(len(f.history), 1),
                              'objective': float(smax[1]), 'same_objective_on_every_rank': bool(smax[1] == smin[1]),
                              'scaling': 'strong'}), flush=True)
    finally:
        dist.destroy_process_group()


def mode_proposal_eval(args):
    """Held-out evaluation of the learned proposal on level-4 shot pairs: iterations and seconds to tolerance."""
    model, rec, heldset = train_proposal(args.train_pairs, args.heldout_pairs, args.train_epochs,
                                                    law=args.momentum_law)
    rec['heldout_eval'] = heldout_registrations(model, heldset, args.heldout_eval)
    print(json.dumps(rec), flush=True)


def ordered_pair_kernel(X, A, lib, nat, ws, wsb, o, sp, flush, peak_fp32, peak_sfu, warmup, reps=20):
    """The same sums through the ordered-pair kernel (pairs_kernel_x<OpK, 128, 8>, the path of K(y,x)a with distinct
    target and source arrays): a copy of x as the targets. Mean device time per sum (CUDA events, L2 flushed before
    each), pairs/s over N^2 and its MUFU / FP32 fractions (6 lane-ops and one ex2 per ordered pair)."""
    import torch
    n = X.shape[0]
    Y = X.clone()
    out = torch.empty_like(X)
    stream = torch.cuda.current_stream()
    ms = []
    for it in range(warmup + reps):
        for s in SIGMAS:
            flush.fill_(1.0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            rc = lib.lddmm_apply_k(nat.ptr(Y), n, nat.ptr(X), nat.ptr(A), n, s, nat.KERNEL_GAUSS, o, nat.ptr(out),
                                   nat.FP32C, ws, wsb, sp)
            e1.record(stream)
            if rc != 0:
                raise RuntimeError(f'lddmm_apply_k failed: {rc}')
            torch.cuda.synchronize()
            if it >= warmup:
                ms.append(e0.elapsed_time(e1))
    t = statistics.mean(ms) * 1e-3
    pps = n * n / t
    return {'kernel': 'pairs_kernel_x<OpK, 128, 8> + finalize_kernel', 'ms_per_sum': t * 1e3, 'pairs_per_s': pps,
            'sfu_frac': pps / 1e12 / peak_sfu, 'fp32_frac': 6 * pps / 1e12 / peak_fp32, 'sums_timed': len(ms),
            'note': 'K(y,x)a with y a distinct copy of x: every ordered pair evaluated; the self-sum path above '
                    'is faster per sum'}


def run_b200(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    from base import _native as nat
    from base.kernelFunctions import Kernel

    torch.cuda.set_device(local_rank)
    x, a_raw = workload()
    n = x.shape[0]
    X = torch.from_numpy(x).cuda()
    K03 = Kernel(name='gauss', sigma=0.3)
    K03.pk_dtype = 'float32'
    A = K03.applyK(X, torch.from_numpy(a_raw).cuda())
    a = A.cpu().numpy()
    lib = nat.lib()
    origin = nat.centroid(X)
    o = nat.origin_arg(origin)
    outs = [torch.empty((n, 3), dtype=torch.float64, device='cuda') for _ in SIGMAS]
    ws, wsb = nat.workspace(n, n, nat.FP32C)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device='cuda')
    stream = torch.cuda.current_stream()
    sp = nat.stream_ptr()

    def step(evs=None):
        for i, s in enumerate(SIGMAS):
            if evs is not None:
                evs[i][0].record(stream)
            rc = lib.lddmm_apply_k(nat.ptr(X), n, nat.ptr(X), nat.ptr(A), n, s, nat.KERNEL_GAUSS, o, nat.ptr(outs[i]),
                                   nat.FP32C, ws, wsb, sp)
            if evs is not None:
                evs[i][1].record(stream)
            if rc != 0:
                raise RuntimeError(f'lddmm_apply_k failed: {rc}')

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    launches = 0
    step_ms, launch_ms = [], []
    with ClockSampler(local_rank) as clk:
        torch.cuda.synchronize()
        clk.mark_start()
        for _ in range(args.steps):
            flush.fill_(1.0)
            evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in SIGMAS]
            step(evs)
            launches += 2 * len(SIGMAS)
            torch.cuda.synchronize()
            ms = [e0.elapsed_time(e1) for e0, e1 in evs]
            launch_ms += ms
            step_ms.append(sum(ms))
        torch.cuda.synchronize()
        clk.mark_end()
    if world > 1:
        dist.barrier()
    total_ms = sum(step_ms)
    t = torch.tensor([total_ms], dtype=torch.float64, device='cuda')
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    total_ms = float(t)
    # pairs of the sum: each unordered pair {k, l} (and k = l) once, as the symmetric kernel evaluates them
    pairs_per_step = len(SIGMAS) * n * (n + 1) // 2
    value = world * pairs_per_step * args.steps / (total_ms * 1e-3)

    # end-to-end through the reference-facing API (numpy in / numpy out)
    K = {s: Kernel(name='gauss', sigma=s) for s in SIGMAS}
    for k in K.values():
        k.pk_dtype = 'float32'
    for _ in range(max(1, args.warmup)):
        for s in SIGMAS:
            K[s].applyK(x, a)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    e2e_ms = []
    for _ in range(args.steps):
        flush.fill_(1.0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for s in SIGMAS:
            r = K[s].applyK(x, a)
        e2e_ms.append(1e3 * (time.perf_counter() - t0))
        launches += 2 * len(SIGMAS)
    te = torch.tensor([sum(e2e_ms)], dtype=torch.float64, device='cuda')
    if world > 1:
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
    e2e_value = world * pairs_per_step * args.steps / (float(te) * 1e-3)
    h2d = len(SIGMAS) * (x.nbytes + a.nbytes)
    d2h = len(SIGMAS) * r.nbytes

    if rank != 0:
        return
    clocks = clk.summary()
    peaks = measured_peaks()
    sm_max = clocks.get('sm_max_mhz') or peaks.get('sm_max_mhz') or 1965.0
    n_sm = torch.cuda.get_device_properties(0).multi_processor_count
    peak_fp32 = n_sm * 128 * sm_max * 1e6 / 1e12          # T lane-ops/s
    peak_sfu = n_sm * 16 * sm_max * 1e6 / 1e12            # T ex2/s
    mean_launch_s = statistics.mean(launch_ms) * 1e-3
    diag, off = sym_pair_counts(n)
    achieved = (OPS_FP32_DIAG * diag + OPS_FP32_OFFDIAG * off) / mean_launch_s / 1e12      # T lane-ops/s
    sfu_frac = (OPS_SFU_PER_PAIR * (diag + off) / mean_launch_s / 1e12) / peak_sfu
    traffic, traffic_source = ncu_traffic()
    cb_targets = args.cpu_targets
    import numba
    cb_threads = numba.config.NUMBA_NUM_THREADS
    numba.set_num_threads(cb_threads)
    cb_val, cb_dt, cb_pairs = cpu_baseline(x, a, cb_targets, cb_threads)
    line = {
        'metric': METRIC, 'value': value, 'unit': 'pairs/s', 'n_gpus': world, 'steps': args.steps,
        'warmup': args.warmup, 'ms_per_step': total_ms / args.steps, 'higher_is_better': True, 'scaling': 'weak',
        'vs_baseline': None, 'dtype': 'f32', 'data': 'synthetic', 'config': config(n),
        'e2e': {'value': e2e_value, 'unit': 'pairs/s', 'h2d_bytes_per_step': int(h2d), 'd2h_bytes_per_step': int(d2h),
                'ms_per_step': float(te) / args.steps, 'api': 'Kernel.applyK(numpy x, numpy a)'},
        'roofline': {'bound': 'fp32', 'achieved': achieved, 'peak': peak_fp32, 'unit': 'T FP32 lane-ops/s',
                     'frac': achieved / peak_fp32, 'sfu_frac': sfu_frac, 'traffic': traffic,
                     'traffic_source': traffic_source, 'algorithmic_bytes': 2 * n * 3 * 8 + n * 3 * 8,
                     'kernel': 'pairs_kernel_symx<OpKSym, 128, 8> + finalize_sym_kernel (timed together per call)',
                     'pairs_evaluated_per_launch': {'ordered_in_block': diag, 'unordered_between_blocks': off},
                     'ops_per_pair': {'fp32_between_blocks': OPS_FP32_OFFDIAG, 'fp32_in_block': OPS_FP32_DIAG,
                                      'sfu': OPS_SFU_PER_PAIR},
                     'peak_source': f'{n_sm} SMs x 128 FP32 lanes x {sm_max:.0f} MHz (nominal pipe peak at the '
                                    f'max SM clock; MEASURED_PEAKS.json has no FP32 figure)'},
        'nm_equivalent_pairs_per_s': value * n / ((n + 1) / 2),
        'cpu_baseline': {'value': cb_val, 'unit': 'pairs/s', 'cores': cb_threads, 'kind': 'port',
                         'sample': f'{cb_pairs:.3g} pairs: blocks of {cb_targets} targets x {n} sources x '
                                   f'{len(SIGMAS)} widths, float64; port: the oracle numba restatement of '
                                   f'ku.applyK_numba without its per-pair temporaries, {cb_dt:.1f} s',
                         'reference_numba_applyK': REFERENCE_NUMBA_APPLYK},
        'clocks': clocks, 'gpu_launches': launches,
        'pairs_per_step': pairs_per_step,
    }
    if world == 1:
        line['ordered_pair_kernel'] = ordered_pair_kernel(X, A, lib, nat, ws, wsb, o, sp, flush, peak_fp32, peak_sfu,
                                                          args.warmup)
    if world == 1 and not args.no_errors:
        line['errors'] = run_errors()
    if world == 1 and not args.no_registration:
        line['registration'] = run_registration(args)
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=200)
    ap.add_argument('--warmup', type=int, default=3)
    ap.add_argument('--impl', default='b200', choices=['b200', 'reference'])
    ap.add_argument('--mode', default='bench',
                    choices=['bench', 'ops', 'registration-profile', 'large-registration', 'proposal-eval',
                             'sharded-registration'])
    ap.add_argument('--cpu-targets', type=int, default=4096)
    ap.add_argument('--ref-targets', type=int, default=2048)
    ap.add_argument('--no-registration', action='store_true', help='skip the end-to-end registration measurement')
    ap.add_argument('--no-errors', action='store_true', help='skip the level-6 FP32-vs-FP64 error statement')
    ap.add_argument('--reg-level', type=int, default=6)
    ap.add_argument('--estar-iters', type=int, default=600, help='iteration cap of the run that derives E*')
    ap.add_argument('--train-pairs', type=int, default=20000, help='pairs generated (trained on + held out)')
    ap.add_argument('--heldout-pairs', type=int, default=2000)
    ap.add_argument('--heldout-eval', type=int, default=8, help='held-out pairs registered with and without the net')
    ap.add_argument('--heldout-seeds', default='1,2', help='bumpy-ellipsoid seeds registered as held-out problems')
    ap.add_argument('--coarse-levels', default='', help='coarse icosphere levels of the warm start (default: per level)')
    ap.add_argument('--momentum-law', default='shapes', choices=['shapes', 'noise'],
                    help='momentum law of the generated training pairs (learnedProposal.generate_pairs)')
    ap.add_argument('--train-epochs', type=int, default=4)
    # mode ops / registration-profile / large-registration
    ap.add_argument('--level', type=int, default=6)
    ap.add_argument('--ops', default='all')
    ap.add_argument('--precision', default='fp32', choices=['fp32', 'fp64'])
    ap.add_argument('--reps', type=int, default=10)
    ap.add_argument('--sigma', type=float, default=0.5)
    ap.add_argument('--sigma-dist', type=float, default=0.2)
    ap.add_argument('--kernel', default='gauss', help="deformation kernel of --mode ops: 'gauss' or 'laplacian:<q>'")
    ap.add_argument('--iters', type=int, default=6)
    ap.add_argument('--warm', default='none', choices=['none', 'multilevel'], help='mode registration-profile')
    ap.add_argument('--fp64-probe-iters', type=int, default=5)
    ap.add_argument('--l7-fp64-full', action='store_true',
                    help='mode large-registration: also run the plain FP64 path to the stopping rule (minutes)')
    args = ap.parse_args()
    world = int(os.environ.get('WORLD_SIZE', '1'))
    rank = int(os.environ.get('RANK', '0'))
    local_rank = int(os.environ.get('LOCAL_RANK', '0'))
    if args.impl == 'reference':
        run_reference(args, rank, world)
        return
    if args.mode == 'sharded-registration':
        mode_sharded_registration(args, rank, world, local_rank)
        return
    if args.mode != 'bench':
        {'ops': mode_ops, 'registration-profile': mode_registration_profile,
         'large-registration': mode_large_registration, 'proposal-eval': mode_proposal_eval}[args.mode](args)
        return
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group('nccl', timeout=datetime.timedelta(seconds=120))
    try:
        run_b200(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == '__main__':
    main()
