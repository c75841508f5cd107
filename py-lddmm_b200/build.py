"""Build the sm_100a shared library `lib/liblddmm_b200.so` (the C-ABI declared in include/lddmm_b200.h).

    python py-lddmm_b200/build.py [--force] [--verbose]

Each .cu in csrc/ is compiled with nvcc for sm_100a (-gencode arch=compute_100a,code=sm_100a, -lineinfo, -O3,
no fast-math: the compensated sums rely on IEEE addition order) and linked into one shared object with the
CUDA runtime statically linked, so that the library loads with nothing but the driver.
"""
import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, 'csrc')
LIBDIR = os.path.join(HERE, 'lib')
OBJDIR = os.path.join(HERE, '_build')
LIBNAME = 'liblddmm_b200.so'
INCLUDE = os.path.join(os.path.dirname(HERE), 'include')

ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']
NVFLAGS = ['-O3', '-lineinfo', '-std=c++17', '-Xcompiler', '-fPIC', '--expt-relaxed-constexpr',
           '-Xptxas', '-warn-spills', f'-I{INCLUDE}']


def nvcc():
    for cand in (os.environ.get('NVCC'), shutil.which('nvcc'), '/usr/local/cuda/bin/nvcc'):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError('nvcc not found')


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith('.cu'))


def headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(('.cuh', '.h'))]
    hs.append(os.path.join(INCLUDE, 'lddmm_b200.h'))
    return hs


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False, ptxas_info=False):
    os.makedirs(LIBDIR, exist_ok=True)
    os.makedirs(OBJDIR, exist_ok=True)
    nv = nvcc()
    hdrs = headers()
    objs, jobs = [], []
    for src in sources():
        obj = os.path.join(OBJDIR, os.path.basename(src)[:-3] + '.o')
        objs.append(obj)
        if force or _stale(obj, [src] + hdrs + [__file__]):
            cmd = [nv] + ARCH + NVFLAGS + (['-Xptxas', '-v'] if ptxas_info else []) + ['-c', src, '-o', obj]
            jobs.append(cmd)

    def run(cmd):
        r = subprocess.run(cmd, capture_output=True, text=True)
        return cmd, r

    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        for cmd, r in ex.map(run, jobs):
            if verbose or r.returncode != 0 or ptxas_info:
                sys.stdout.write(' '.join(cmd) + '\n' + r.stdout + r.stderr)
            if r.returncode != 0:
                raise RuntimeError(f'nvcc failed for {cmd[-3]}')
    lib = os.path.join(LIBDIR, LIBNAME)
    if force or jobs or _stale(lib, objs):
        cmd = [nv] + ARCH + ['-shared', '-Xcompiler', '-fPIC', '-cudart', 'static', '-o', lib] + objs
        r = subprocess.run(cmd, capture_output=True, text=True)
        if verbose or r.returncode != 0:
            sys.stdout.write(' '.join(cmd) + '\n' + r.stdout + r.stderr)
        if r.returncode != 0:
            raise RuntimeError('link failed')
    return lib


if __name__ == '__main__':
    ap = argparse.ArgumentParser()
    ap.add_argument('--force', action='store_true')
    ap.add_argument('--verbose', action='store_true')
    ap.add_argument('--ptxas-info', action='store_true')
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose, ptxas_info=a.ptxas_info))
