"""Generate the golden fixtures in this folder by running the reference py-lddmm itself (float64 numba path).

Usage (in a container where the reference tree is mounted):
    python tests/golden/make_golden.py --ref <the reference's py-lddmm directory>

The reference's module-level imports need four shims; none of them changes a reference file:
  1. `keopscore` stub with `config.config.use_cuda = False` (hard import at base/kernelFunctions_util.py:13,
     base/surfaceDistances.py:5) -- selects the `_numba` / `_numpy` CPU implementations;
  2. `scipy.optimize.linesearch` -> `scipy.optimize._linesearch` (import at base/linesearch.py:2);
  3. `np.Inf = np.inf` (numpy 2 removed it; used at base/basicMatching.py:55);
  4. empty stand-ins for optional modules imported by the matching classes (pyfftw, skimage, vtk, h5py,
     matplotlib, mpl_toolkits, pygalmesh) and aliases for the module names `base.surfaceDistancess`
     (sic, base/surfaceMatching.py:9) and top-level `pointset_distances` (base/surfaceMatching.py:14).

Every fixture stores its inputs next to the reference outputs, so the tests never regenerate inputs.
"""
import argparse
import importlib.util
import logging
import os
import sys
import tempfile
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))


def install_shims():
    kc = types.ModuleType('keopscore')
    kc.config = types.SimpleNamespace(config=types.SimpleNamespace(use_cuda=False))
    sys.modules['keopscore'] = kc
    import scipy.optimize
    import scipy.optimize._linesearch as ls
    sys.modules['scipy.optimize.linesearch'] = ls
    scipy.optimize.linesearch = ls
    np.Inf = np.inf

    class _Any(types.ModuleType):
        def __getattr__(self, name):
            if name.startswith('__'):
                raise AttributeError(name)
            m = _Any(self.__name__ + '.' + name)
            sys.modules[m.__name__] = m
            return m

        def __call__(self, *a, **k):
            return _Any('call')

    for name in ['pyfftw', 'pyfftw.interfaces', 'pyfftw.interfaces.numpy_fft', 'skimage', 'skimage.measure',
                 'skimage.morphology', 'skimage.segmentation', 'skimage.filters', 'skimage.draw',
                 'vtk', 'vtk.util', 'vtk.util.numpy_support', 'h5py', 'matplotlib', 'matplotlib.pyplot',
                 'matplotlib.colors', 'matplotlib.cm', 'mpl_toolkits', 'mpl_toolkits.mplot3d',
                 'mpl_toolkits.mplot3d.art3d', 'pygalmesh', 'meshpy', 'meshpy.triangle', 'nibabel',
                 'imageio', 'PIL', 'PIL.Image', 'tqdm']:
        if name not in sys.modules:
            try:
                importlib.import_module(name)
            except Exception:
                sys.modules[name] = _Any(name)


def load_shapes():
    spec = importlib.util.spec_from_file_location(
        'syntheticShapes', os.path.join(REPO, 'py-lddmm_b200', 'base', 'syntheticShapes.py'))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def smooth_momenta(kf, shapes, x, rng, sigma_smooth, sigma_def=0.5, vmax=0.3):
    """The package's normalised recipe (syntheticShapes.smooth_momenta) evaluated with the reference's Kernel."""
    return shapes.smooth_momenta(x, rng, lambda y_, x_, a_, s: kf.Kernel(name='gauss', sigma=s).applyK(x_, a_, firstVar=y_),
                                 sigma_smooth=sigma_smooth, sigma_def=sigma_def, vmax=vmax)


def kernel_fixtures(kf, shapes, out):
    """Fixtures for Kernel.applyK / applyDiffKT / applyDDiffK11and12 / applyDiffK1and2 / applyKTensor /
    applyDivergence / applyDiffKmat / applyK(matrixWeights) (base/kernelFunctions.py:452-674)."""
    rng = np.random.default_rng(1234)
    for level in (2, 3):
        x, _ = shapes.icosphere(level)
        n = x.shape[0]
        y = shapes.bumpy_ellipsoid(x, seed=5)[: n // 3 + 7] * 1.05
        for sigma in (0.25, 0.5):
            K = kf.Kernel(name='gauss', sigma=sigma)
            a = rng.normal(size=(n, 3))
            p = rng.normal(size=(n, 3))
            q = rng.normal(size=(n, 3))
            rec = dict(x=x, y=y, a=a, p=p, q=q, sigma=sigma, regweight=0.7)
            rec['applyK'] = K.applyK(x, a)
            rec['applyK_cross'] = K.applyK(x, a, firstVar=y)
            rec['applyDiffKT'] = K.applyDiffKT(x, p, a)
            rec['applyDiffKT_cross'] = K.applyDiffKT(x, p[: y.shape[0]], a, firstVar=y)
            rec['applyDiffKT_sym'] = K.applyDiffKT(x, p, a, sym=True)
            rec['applyDiffKT_lddmm'] = K.applyDiffKT(x, p, a, lddmm=True, regweight=0.7)
            rec['applyDDiffK11and12'] = K.applyDDiffK11and12(x, a, q, p)
            rec['applyDiffK1and2'] = K.applyDiffK1and2(x, p, a)
            rec['applyDivergence'] = K.applyDivergence(x, a)
            rec['applyDivergence_cross'] = K.applyDivergence(x, a, firstVar=y)
            w_t = np.abs(rng.normal(size=n)) + 0.1
            bt = rng.normal(size=(n, 3))
            rec['ay'] = w_t
            rec['betay'] = bt
            rec['applyKTensor'] = K.applyKTensor(x, w_t, w_t, bt, bt)
            rec['applyKTensor_cross'] = K.applyKTensor(x, w_t[: y.shape[0]], w_t, bt[: y.shape[0]], bt, firstVar=y)
            if level == 2:
                beta = rng.normal(size=(n, n))
                u = rng.normal(size=(n, n, 3))
                rec['beta'] = beta
                rec['u'] = u
                rec['applyDiffKmat'] = K.applyDiffKmat(x, beta)
                rec['applyK_mat'] = K.applyK(x, u, matrixWeights=True)
            out[f'kernels_L{level}_s{sigma}'] = rec


def shooting_fixtures(kf, evol, shapes, out):
    """landmarkDirectEvolutionEuler / landmarkHamiltonianGradient (base/pointEvolution.py:88-236) and
    secondOrderEvolution / secondOrderGradient (base/pointEvolution.py:385-618)."""
    rng = np.random.default_rng(99)
    x0, _ = shapes.icosphere(2)
    K = kf.Kernel(name='gauss', sigma=0.5)
    T = 10
    at = np.stack([smooth_momenta(kf, shapes, x0, rng, 0.3, vmax=0.3) for _ in range(T)])
    px1 = rng.normal(0.0, 0.5, size=x0.shape)
    st = evol.landmarkDirectEvolutionEuler(x0, at, K)
    dat, xt, pxt = evol.landmarkHamiltonianGradient(x0, at, px1, K, 0.8, getCovector=True)
    out['first_order_L2'] = dict(x0=x0, at=at, px1=px1, sigma=0.5, regweight=0.8,
                                 xt=st['xt'], dat=dat, xt_grad=xt, pxt=pxt)
    a0 = smooth_momenta(kf, shapes, x0, rng, 0.4, vmax=0.3)
    fw = evol.secondOrderEvolution(x0, a0, K, 0.1)
    pa1 = rng.normal(0.0, 0.2, size=x0.shape)
    g = evol.secondOrderGradient(x0, a0, px1, pa1, K, 0.1)
    out['second_order_L2'] = dict(x0=x0, a0=a0, px1=px1, pa1=pa1, sigma=0.5, timeStep=0.1,
                                  xt=fw['xt'], at=fw['at'], da0=g['da0'], pxt=g['pxt'], pat=g['pat'])


def epdiff_fixtures(kf, evol, shapes, out):
    """landmarkEPDiff (base/pointEvolution.py:320-382) with a point set and normals. (withJacobian=True raises in
    the reference: line 366 adds an (N,1) divergence to an (N,) slice.)"""
    rng = np.random.default_rng(77)
    x0, _ = shapes.icosphere(2)
    K = kf.Kernel(name='gauss', sigma=0.5)
    a0 = smooth_momenta(kf, shapes, x0, rng, 0.4, vmax=0.3)
    y0 = shapes.bumpy_ellipsoid(x0, seed=3)[:40] * 0.9
    n0 = rng.normal(size=x0.shape)
    xt, at, yt, nt = evol.landmarkEPDiff(8, x0, a0, K, withNormals=n0, withPointSet=y0)
    out['epdiff_L2'] = dict(x0=x0, a0=a0, y0=y0, n0=n0, sigma=0.5, T=8, xt=xt, at=at, yt=yt, nt=nt)


def laplacian_fixtures(kf, evol, shapes, out):
    """The same operators and both shooting variants with the reference's Laplacian kernel
    (KernelSpec(name='laplacian', order=q), base/kernelFunctions.py:363-368; lap_fun* at
    base/kernelFunctions_util.py:92-96, 197-203, 239-243, 309-314)."""
    rng = np.random.default_rng(4321)
    x, _ = shapes.icosphere(2)
    n = x.shape[0]
    y = shapes.bumpy_ellipsoid(x, seed=5)[: n // 3 + 7] * 1.05
    for order in (1, 3, 4):
        K = kf.Kernel(name='laplacian', sigma=0.5, order=order)
        a = rng.normal(size=(n, 3))
        p = rng.normal(size=(n, 3))
        q = rng.normal(size=(n, 3))
        rec = dict(x=x, y=y, a=a, p=p, q=q, sigma=0.5, order=order, regweight=0.7)
        rec['applyK'] = K.applyK(x, a)
        rec['applyK_cross'] = K.applyK(x, a, firstVar=y)
        rec['applyDiffKT'] = K.applyDiffKT(x, p, a)
        rec['applyDiffKT_cross'] = K.applyDiffKT(x, p[: y.shape[0]], a, firstVar=y)
        rec['applyDiffKT_sym'] = K.applyDiffKT(x, p, a, sym=True)
        rec['applyDiffKT_lddmm'] = K.applyDiffKT(x, p, a, lddmm=True, regweight=0.7)
        rec['applyDDiffK11and12'] = K.applyDDiffK11and12(x, a, q, p)
        rec['applyDiffK1and2'] = K.applyDiffK1and2(x, p, a)
        rec['applyDivergence'] = K.applyDivergence(x, a)
        out[f'laplacian_L2_o{order}'] = rec
    K = kf.Kernel(name='laplacian', sigma=0.5, order=3)
    T = 10
    at = np.stack([smooth_momenta(kf, shapes, x, rng, 0.3, vmax=0.3) for _ in range(T)])
    px1 = rng.normal(0.0, 0.5, size=x.shape)
    st = evol.landmarkDirectEvolutionEuler(x, at, K)
    dat, xt, pxt = evol.landmarkHamiltonianGradient(x, at, px1, K, 0.8, getCovector=True)
    a0 = smooth_momenta(kf, shapes, x, rng, 0.4, vmax=0.3)
    fw = evol.secondOrderEvolution(x, a0, K, 0.1)
    pa1 = rng.normal(0.0, 0.2, size=x.shape)
    g = evol.secondOrderGradient(x, a0, px1, pa1, K, 0.1)
    out['laplacian_shooting_L2_o3'] = dict(x0=x, at=at, a0=a0, px1=px1, pa1=pa1, sigma=0.5, order=3, regweight=0.8,
                                           timeStep=0.1, fo_xt=st['xt'], fo_dat=dat, fo_pxt=pxt, xt=fw['xt'],
                                           at_so=fw['at'], da0=g['da0'], pxt=g['pxt'], pat=g['pat'])


def data_term_fixtures(kf, sd, surf, shapes, out):
    """varifoldNorm0/Def/Gradient, currentNorm0/Def/Gradient, measureNorm0/Def/Gradient
    (base/surfaceDistances.py:22-573)."""
    rng = np.random.default_rng(7)
    for level in (2, 3):
        x0, faces = shapes.icosphere(level)
        x1 = shapes.bumpy_ellipsoid(x0, seed=0)
        xdef = x0 * 1.1 + 0.02 * rng.normal(size=x0.shape)
        wts = 0.5 + rng.random(x0.shape[0])
        for sigma in (0.2, 0.3):
            Kd = kf.Kernel(name='gauss', sigma=sigma)
            fv1 = surf.Surface(surf=(faces, x1))
            fvd = surf.Surface(surf=(faces, xdef))
            fvw = surf.Surface(surf=(faces, xdef), weights=wts)
            rec = dict(x1=x1, xdef=xdef, faces=faces, weights=wts, sigma=sigma)
            rec['varifoldNorm0'] = sd.varifoldNorm0(fv1, Kd)
            rec['varifoldNormDef'] = sd.varifoldNormDef(fvd, fv1, Kd)
            rec['varifoldNormGradient'] = sd.varifoldNormGradient(fvd, fv1, Kd)
            rec['varifoldNormDef_w'] = sd.varifoldNormDef(fvw, fv1, Kd)
            # with_weights=True raises under numpy 2 in the reference (base/surfaceDistances.py:463-465 adds a
            # length-1 array into a scalar slot), so only the vertex gradient of the weighted surface is pinned.
            rec['varifoldNormGradient_w'] = sd.varifoldNormGradient(fvw, fv1, Kd)
            rec['currentNorm0'] = sd.currentNorm0(fv1, Kd)
            rec['currentNormDef'] = sd.currentNormDef(fvd, fv1, Kd)
            rec['currentNormGradient'] = sd.currentNormGradient(fvd, fv1, Kd)
            rec['measureNorm0'] = sd.measureNorm0(fv1, Kd)
            rec['measureNormDef'] = sd.measureNormDef(fvd, fv1, Kd)
            rec['measureNormGradient'] = sd.measureNormGradient(fvd, fv1, Kd)
            out[f'data_L{level}_s{sigma}'] = rec


def matching_fixtures(kf, surf, sm_mod, so_mod, shapes, out, iters, laplacian=False):
    """End-to-end runs of SurfaceMatching / SecondOrderSurfaceMatching (base/surfaceMatching.py:75,
    base/secondOrderSurfaceMatching.py:41) with BFGS (base/bfgs.py:55): objective at iteration 0, the first
    gradient and the objective after each of `iters` iterations. With `laplacian`, the deformation kernel is the
    reference's Laplacian kernel of order 3 (fixtures matching_*_lap_L2)."""
    x0, faces = shapes.icosphere(2)
    x1 = shapes.bumpy_ellipsoid(x0, seed=0)
    tag = '_lap' if laplacian else ''
    for name, cls in (('first', sm_mod.SurfaceMatching), ('second', so_mod.SecondOrderSurfaceMatching)):
        objs = []
        with tempfile.TemporaryDirectory() as tmp:
            fv0 = surf.Surface(surf=(faces, x0))
            fv1 = surf.Surface(surf=(faces, x1))
            opts = dict(outputDir=tmp, mode='normal', maxIter=iters, affine='none', regWeight=1.0,
                        KparDiff=(kf.Kernel(name='laplacian', sigma=0.5, order=3) if laplacian
                                  else kf.Kernel(name='gauss', sigma=0.5)),
                        KparDist=('gauss', 0.3), sigmaError=1.0,
                        errorType='varifold', pk_dtype='float64', algorithm='bfgs', timeStep=0.1, saveRate=10 ** 6,
                        verb=False)
            f = cls(Template=fv0, Target=fv1, options=opts)
            obj0 = f.objectiveFun()
            g0 = f.getGradient(f.gradCoeff)
            orig_end = f.endOfIteration

            def eoi(*a, **k):
                r = orig_end(*a, **k)
                objs.append(float(f.obj))
                return r
            f.endOfIteration = eoi
            f.optimizeMatching()
            key = 'at' if name == 'first' else 'a0'
            out[f'matching_{name}{tag}_L2'] = dict(x0=x0, x1=x1, faces=faces, obj0=obj0, grad0=g0[key],
                                              objs=np.array(objs), control=f.control[key])


def save(out):
    for name, rec in out.items():
        path = os.path.join(HERE, name + '.npz')
        np.savez_compressed(path, **{k: np.asarray(v) for k, v in rec.items()})
        print('wrote', path, os.path.getsize(path))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--ref', required=True, help='the py-lddmm directory of the reference tree')
    ap.add_argument('--only', default='')
    ap.add_argument('--iters', type=int, default=5)
    args = ap.parse_args()
    logging.disable(logging.WARNING)
    install_shims()
    sys.path.insert(0, args.ref)
    sys.path.insert(0, os.path.join(args.ref, 'base'))
    from base import kernelFunctions as kf, pointEvolution as evol, surfaceDistances as sd, surfaces as surf
    sys.modules['base.surfaceDistancess'] = sd
    import base.pointset_distances as psd
    sys.modules['pointset_distances'] = psd
    shapes = load_shapes()
    out = {}
    only = args.only.split(',') if args.only else ['kernels', 'shooting', 'epdiff', 'laplacian', 'data',
                                                   'matching', 'matching_lap']
    if 'kernels' in only:
        kernel_fixtures(kf, shapes, out)
    if 'shooting' in only:
        shooting_fixtures(kf, evol, shapes, out)
    if 'epdiff' in only:
        epdiff_fixtures(kf, evol, shapes, out)
    if 'laplacian' in only:
        laplacian_fixtures(kf, evol, shapes, out)
    if 'data' in only:
        data_term_fixtures(kf, sd, surf, shapes, out)
    if 'matching' in only:
        from base import surfaceMatching as sm_mod, secondOrderSurfaceMatching as so_mod
        matching_fixtures(kf, surf, sm_mod, so_mod, shapes, out, args.iters)
    if 'matching_lap' in only:
        from base import surfaceMatching as sm_mod, secondOrderSurfaceMatching as so_mod
        matching_fixtures(kf, surf, sm_mod, so_mod, shapes, out, args.iters, laplacian=True)
    save(out)


if __name__ == '__main__':
    main()
