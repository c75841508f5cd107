"""Benchmark of the B200 point-set hot path: Gaussian kernel pair-evaluations per second.

Workload ("L6 kernel sums", the deformation-kernel sums of the level-6 registration): source vertices of the
level-6 icosphere (N = M = 40,962), smoothed momenta a = K_0.3 (N(0, 0.1^2)), Gaussian widths sigma = 0.25
and 0.5. One step = K(x, x) a for both widths (2 * N^2 pair evaluations), FP32 pair arithmetic with
compensated accumulation and FP64 outputs.

  value     pairs/s with inputs resident in HBM, device-timed (CUDA events per step, L2 flushed between steps
            by writing a 256 MiB buffer; the flush is outside the timed events)
  e2e       the same step through the reference-facing API `Kernel.applyK(x, a)` with numpy (host) arrays:
            host->device copy of x and a, the kernels, device->host copy of the result, every step
  roofline  the pair kernel against the MUFU (ex2) pipe, its binding pipe: 1 SFU op + 6 FP32 lane-ops per pair
            (expanded-distance form: 3 FMAs for |x|^2 - 2 y.x about the target block's centre, one ex2, 3 FMAs
            accumulating K a); peak = 148 SMs x 16 MUFU lanes x max SM clock (the FP32 fraction is reported
            beside it against 148 x 128 FP32 lanes x max SM clock)
  cpu_baseline  the CPU oracle (numba, float64, all host threads) on a bounded sample of the same sums

`--impl reference` times the CPU implementation of the same sums (the oracle restatement of the reference's
numba kernels, all host threads) and prints the same metric with "impl": "reference".

  registration  (1 GPU) seconds per registration pair to reach 1e-3 relative energy of the FP64 plain optimum on
            the level-6 problem: plain FP64 path, FP32 path, FP32 path + learned warm start (the other half of the
            headline metric), and the level-4 problem run for 50 BFGS iterations on the FP64 path (both matching
            classes; the case the reference itself runs on the CPU); skipped with --no-registration

Multi-GPU (torchrun): every rank runs the same workload on its own GPU (independent replicas, weak scaling);
times are the max over ranks; value = pairs of all ranks / that time.
"""
import argparse
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
OPS_FP32_PER_PAIR = 6
OPS_SFU_PER_PAIR = 1
METRIC = 'Gauss kernel pairs/s'


def workload():
    from base.syntheticShapes import icosphere
    x, _ = icosphere(LEVEL)
    rng = np.random.default_rng(1)
    a_raw = rng.normal(0.0, 0.1, size=x.shape)
    return x, a_raw


def config(n):
    return {'workload': 'L6 kernel sums: K(x,x)a, icosphere level 6, N=M=%d, sigma in %s, smoothed momenta' % (
        n, list(SIGMAS)), 'level': LEVEL, 'n_points': n, 'sigmas': list(SIGMAS), 'op': 'applyK (Gaussian)',
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


def ncu_traffic():
    """dram bytes per launch of the pair kernel from the committed ncu summary (profiles/)."""
    p = os.path.join(REPO, 'profiles', 'applyk_pairs_L6_ncu.json')
    try:
        d = json.load(open(p))
        return d.get('dram_bytes_per_launch')
    except Exception:
        return None


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
                                       f'(oracle numba restatement of ku.applyK_numba, float64)'},
            'e2e': {'value': value, 'unit': 'pairs/s', 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0},
            'setup_s': setup}
    print(json.dumps(line), flush=True)


# E* of the L6 registration below: FP64 plain path (pk_dtype float64, zero initial momentum) run to the reference's
# BFGS stopping rule (108 iterations, |obj - obj_old| < 1e-7); `--recompute-estar` re-derives it.
L6_ESTAR = 0.12269117945467034


def run_registration(args):
    """Seconds per registration pair to reach (E - E*)/E* <= 1e-3 on the level-6 icosphere -> bumpy ellipsoid problem
    (Gaussian sigma 0.5, varifold sigma 0.2, T = 20, sigmaError 1, BFGS): plain FP64 path vs FP32 path vs FP32 path with
    the learned warm start (network trained here, at level 4, on pairs generated by shooting)."""
    import torch
    from base import learnedProposal as lp
    from base.kernelFunctions import Kernel
    from base.surfaceMatching import SecondOrderSurfaceMatching
    from base.surfaces import Surface
    from base.syntheticShapes import icosphere, bumpy_ellipsoid
    level = args.reg_level
    x0, F = icosphere(level)
    x1 = bumpy_ellipsoid(x0, seed=0)

    def solve(dtype, target=None, model=None, maxIter=600):
        K = Kernel(name='gauss', sigma=0.5)
        K.pk_dtype = dtype
        opts = dict(maxIter=maxIter, affine='none', regWeight=1.0, KparDiff=K, KparDist=('gauss', 0.2), sigmaError=1.0,
                    errorType='varifold', pk_dtype=dtype, algorithm='bfgs', timeStep=0.05, verb=False,
                    targetObjective=target)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        f = SecondOrderSurfaceMatching(Template=Surface(surf=(F, x0)), Target=Surface(surf=(F, x1)), options=opts)
        used = lp.warm_start(f, model, scales=(0.5, 0.75, 1.0)) if model is not None else None
        f.optimizeMatching()
        torch.cuda.synchronize()
        return f, time.perf_counter() - t0, used

    res = {'problem': f'icosphere L{level} ({x0.shape[0]} vertices) -> bumpy ellipsoid, sigma 0.5 / varifold 0.2, '
                      'T=20, sigmaError 1, BFGS', 'criterion': '(E - E*)/E* <= 1e-3'}
    if args.recompute_estar or level != 6:
        f64, t, _ = solve('float64')
        estar = f64.history[-1]
        res['estar_run'] = {'iters': len(f64.history), 's': t}
    else:
        estar = L6_ESTAR
    res['estar'] = estar
    target = estar * (1 + 1e-3)
    t0 = time.perf_counter()
    xs, Fs = icosphere(4)
    feats, labels, _, n4 = lp.generate_pairs(xs, Fs, args.train_pairs, seed=0, timeStep=0.1)
    model = lp.MomentumProposal(seed=0)
    ntr = int(0.9 * args.train_pairs)
    hist = lp.train(model, feats[:ntr], labels[:ntr], n4, epochs=args.train_epochs, batch_pairs=16, lr=2e-3)
    with torch.no_grad():
        y = model.forward(feats[ntr:].reshape(-1, lp.IN_DIM)).reshape(-1, feats.shape[1], lp.OUT_DIM)[:, :n4, :3]
    res['proposal'] = {'train_pairs': ntr, 'heldout_pairs': args.train_pairs - ntr, 'epochs': args.train_epochs,
                       'train_s': time.perf_counter() - t0, 'loss_first_last': [hist[0], hist[-1]],
                       'heldout_label_rel_err': float((y - labels[ntr:, :n4]).norm() / labels[ntr:, :n4].norm())}
    for name, dtype, model_ in (('plain_fp64', 'float64', None), ('plain_fp32', 'float32', None),
                                ('learned_fp32', 'float32', model)):
        f, t, used = solve(dtype, target=target, model=model_)
        f.resetPK('float64')
        f.obj = None
        e = f.objectiveFun()
        res[name] = {'s_per_pair': t, 'iters': len(f.history), 'reached': bool(f.reached_target),
                     'rel_energy_fp64': (e - estar) / abs(estar)}
        if used is not None:
            res[name].update({'proposal_used': used[0], 'obj_proposal': used[1], 'obj_zero': used[2]})
    res['speedup_learned_vs_plain_fp64'] = res['plain_fp64']['s_per_pair'] / res['learned_fp32']['s_per_pair']
    res['speedup_plain_fp32_vs_plain_fp64'] = res['plain_fp64']['s_per_pair'] / res['plain_fp32']['s_per_pair']
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
    pairs_per_step = len(SIGMAS) * n * n
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
    achieved = n * n * OPS_SFU_PER_PAIR / mean_launch_s / 1e12
    fp32_frac = (n * n * OPS_FP32_PER_PAIR / mean_launch_s / 1e12) / peak_fp32
    traffic = ncu_traffic()
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
        'roofline': {'bound': 'sfu', 'achieved': achieved, 'peak': peak_sfu, 'unit': 'T ex2/s',
                     'frac': achieved / peak_sfu, 'fp32_frac': fp32_frac, 'traffic': traffic,
                     'kernel': 'pairs_kernel_x<OpK, 128, 8> + finalize_kernel (timed together per call)',
                     'ops_per_pair': {'fp32': OPS_FP32_PER_PAIR, 'sfu': OPS_SFU_PER_PAIR},
                     'peak_source': f'{n_sm} SMs x 16 MUFU lanes x {sm_max:.0f} MHz (nominal pipe peak at the '
                                    f'max SM clock; MEASURED_PEAKS.json has no MUFU or FP32 figure)'},
        'cpu_baseline': {'value': cb_val, 'unit': 'pairs/s', 'cores': cb_threads, 'kind': 'port',
                         'sample': f'{cb_pairs:.3g} pairs: blocks of {cb_targets} targets x {n} sources x '
                                   f'{len(SIGMAS)} widths, float64 numba oracle, {cb_dt:.1f} s'},
        'clocks': clocks, 'gpu_launches': launches,
        'pairs_per_step': pairs_per_step,
    }
    if world == 1 and not args.no_registration:
        line['registration'] = run_registration(args)
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=200)
    ap.add_argument('--warmup', type=int, default=3)
    ap.add_argument('--impl', default='b200', choices=['b200', 'reference'])
    ap.add_argument('--cpu-targets', type=int, default=4096)
    ap.add_argument('--ref-targets', type=int, default=2048)
    ap.add_argument('--no-registration', action='store_true', help='skip the end-to-end registration measurement')
    ap.add_argument('--recompute-estar', action='store_true')
    ap.add_argument('--reg-level', type=int, default=6)
    ap.add_argument('--train-pairs', type=int, default=2000)
    ap.add_argument('--train-epochs', type=int, default=20)
    args = ap.parse_args()
    world = int(os.environ.get('WORLD_SIZE', '1'))
    rank = int(os.environ.get('RANK', '0'))
    local_rank = int(os.environ.get('LOCAL_RANK', '0'))
    if args.impl == 'reference':
        run_reference(args, rank, world)
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
