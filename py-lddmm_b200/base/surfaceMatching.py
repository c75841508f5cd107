"""Drop-in surface matching drivers with device-resident state (reference: base/surfaceMatching.py:75-1590,
base/secondOrderSurfaceMatching.py:41, base/pointSetMatching.py, base/basicMatching.py).

`SurfaceMatching` (first-order LDDMM, controls a_t, t < T) and `SecondOrderSurfaceMatching` (geodesic shooting
from a_0) keep the reference's options dictionary, the optimiser protocol (objectiveFun, updateTry, getGradient,
acceptVarTry, dotProduct_euclidean, addProd, prod, copyDir, randomDir, startOfIteration, endOfIteration) and
`optimizeMatching()` (L-BFGS, memory 50, weak Wolfe). Controls, trajectories and covectors are float64 CUDA
tensors; every kernel sum runs in the sm_100a library; the objective and the dot products are FP64 device
reductions read back as Python floats for the line-search comparisons.

Differences from the reference, by design:
  * the trajectory computed for a line-search trial is reused by the gradient at the accepted step (the reference
    shoots forward again inside every gradient, base/pointEvolution.py:516-519 and base/surfaceMatching.py:757);
  * the first-order kinetic energy sum_t a_t.K(x_t)a_t is read from the shooting kernels' epilogue instead of a
    second K(x_t)a_t per time step (base/surfaceMatching.py:546-548);
  * affine parts, landmarks, symmetric / unreduced / SGD variants are not implemented; of the file output, the
    result record of `saveHdf5` is written as an .npz archive with the same keys (h5py is not available).
"""
import ctypes
import logging
import time
from copy import deepcopy

import numpy as np
import torch

from . import _native as nat
from . import bfgs as _bfgs
from . import pointEvolution as evol
from .kernelFunctions import Kernel
from .surfaceDistances import SurfaceDataTerm
from .surfaces import Surface


class Control(dict):
    pass


class TargetReached(Exception):
    """Raised at the end of an iteration whose objective is at or below options['targetObjective']."""


class State(dict):
    pass


def _make_kernel(spec, default_sigma):
    if isinstance(spec, Kernel):
        return spec
    if spec is None:
        return Kernel(name='gauss', sigma=default_sigma)
    if isinstance(spec, (list, tuple)):
        return Kernel(name=spec[0], sigma=spec[1])
    raise TypeError('kernel must be a Kernel or a (name, sigma) tuple')


class _DeviceMatching:
    control_key = None

    def getDefaultOptions(self):
        return {'timeStep': 0.1, 'algorithm': 'bfgs', 'unreduced': False, 'Wolfe': True, 'burnIn': 10,
                'epsInit': 1., 'KparDiff': None, 'KparDist': None, 'pk_dtype': 'float32', 'sigmaError': 1.0,
                'errorType': 'measure', 'vfun': None, 'maxIter': 1000, 'regWeight': 1.0, 'affine': None,
                'affineKernel': False, 'testGradient': False, 'Landmarks': None, 'saveFile': 'evolution',
                'saveRate': 10, 'mode': 'normal', 'verb': True, 'pplot': False, 'outputDir': '.',
                'symmetric': False, 'internalCost': None, 'lineSearch': 'Weak_Wolfe', 'gradTol': -1.,
                'gradLB': 0.001, 'initialMomentum': None, 'targetObjective': None, 'processGroup': None,
                'warmStart': None}

    def __init__(self, Template=None, Target=None, options=None):
        self.options = self.getDefaultOptions()
        if options is not None:
            self.options.update(options)
        o = self.options
        if o['affine'] not in (None, 'none'):
            raise NotImplementedError('affine components are not implemented')
        if o['Landmarks'] is not None or o['symmetric'] or o['unreduced'] or o['internalCost'] is not None:
            raise NotImplementedError('landmarks / symmetric / unreduced / internal-cost variants are not implemented')
        if o['algorithm'] not in ('bfgs',):
            raise NotImplementedError("algorithm='bfgs' is implemented")
        if o['mode'] == 'debug':
            o['testGradient'] = True
            o['pk_dtype'] = 'float64'
        self.fv0 = Surface(surf=Template)
        self.fv1 = Surface(surf=Target)
        self.fvDef = Surface(surf=self.fv0)
        self.dim = 3
        o['KparDiff'] = _make_kernel(o['KparDiff'], 6.5)
        o['KparDist'] = _make_kernel(o['KparDist'], 2.5)
        self.Kdiff_dtype = o['pk_dtype']
        self.resetPK(o['pk_dtype'])
        kind = o['errorType']
        if kind not in ('varifold', 'current', 'measure'):
            raise NotImplementedError(f"errorType '{kind}' is not implemented")
        if o['vfun'] is not None:
            raise NotImplementedError('only the default varifold weight is implemented')
        w0 = np.asarray(self.fv0.weights, dtype=np.float64)
        w1 = np.asarray(self.fv1.weights, dtype=np.float64)
        self.data = SurfaceDataTerm(self.fv0.faces, self.fv1.vertices, self.fv1.faces, o['KparDist'], kind=kind,
                                    weights=None if np.all(w0 == 1) else w0, target_weights=None if np.all(w1 == 1)
                                    else w1, nv=self.fv0.vertices.shape[0])
        self.x0 = nat.as_device(self.fv0.vertices)
        self.npt = self.x0.shape[0]
        self.origin = nat.centroid(self.x0)
        self.Tsize = int(round(1.0 / o['timeStep']))
        self.sigma2 = o['sigmaError'] ** 2
        self.euclideanGradient = True
        self.gradCoeff = 1.
        self.gradEps = o['gradTol']
        self.burnIn = o['burnIn']
        self.obj = None
        self.objTry = None
        self.reset = False
        self.iter = 0
        self.pkBuffer = 0
        self.history = []
        self.times = []
        self._last_trial = None
        self._grad_cache = None
        self._control_version = 0
        self.control = Control()
        self.controlTry = Control()
        self.state = State()
        self.stateTry = None
        self.initialize_variables()

    # ------------------------------------------------------------------ precision switching
    def resetPK(self, newType=None):
        t = self.Kdiff_dtype if newType is None else newType
        self.options['KparDiff'].pk_dtype = t
        self.options['KparDist'].pk_dtype = t
        if hasattr(self, 'data'):
            self.data.precision = nat.FP64 if t == 'float64' else nat.FP32C
        self.pkBuffer = 0

    def startOfIteration(self):
        if self.reset:
            logging.info('restart after a failed line search: kernel sums now in float64')
            self.resetPK('float64')

    # ------------------------------------------------------------------ data term
    def dataTerm(self, xdef):
        return self.data.energy(xdef)[0] / self.sigma2

    def endPointGradient(self, xdef):
        return self.data.gradient(xdef) / self.sigma2

    # ------------------------------------------------------------------ optimiser protocol
    def getVariable(self):
        return self.control

    def objectiveFun(self):
        if self.obj is None:
            self.obj0 = self.data.norm0() / self.sigma2
            objDef, self.state = self.objectiveFunDef(self.control, withTrajectory=True)
            self.obj = float(self.obj0 + objDef + self.dataTerm(self.state['xt'][-1]))
        return self.obj

    def updateTry(self, dr, eps, objRef=None):
        controlTry = Control()
        for k, v in dr.items():
            if v is not None and self.control.get(k) is not None:
                controlTry[k] = self.control[k] - eps * v
        objDef, st = self.objectiveFunDef(controlTry, withTrajectory=True)
        objTry = float(self.obj0 + objDef + self.dataTerm(st['xt'][-1]))
        # the line search asks for the gradient at the trial point it just evaluated: keep its trajectory
        self._last_trial = (dr, float(eps), self._control_version, controlTry, st, self._control_key())
        if np.isnan(objTry):
            return 1e500
        if objRef is None or objTry < objRef:
            self.controlTry = controlTry
            self.stateTry = st
            self.objTry = objTry
        return objTry

    def getGradient(self, coeff=1.0, update=None):
        """The optimiser's gradient at the current control, or at control - update[1] * update[0]. The gradient at
        the current control is kept until the control, its tensors or the precision change: optimizeMatching asks
        for it once for the gradient threshold and BFGS again for its first step."""
        if update is not None:
            return self._gradient(coeff, update)
        key = (self._control_version, self._control_key(), float(coeff), str(self.options['KparDiff'].pk_dtype))
        if self._grad_cache is None or self._grad_cache[0] != key:
            self._grad_cache = (key, self._gradient(coeff))
        return self._grad_cache[1]

    def acceptVarTry(self):
        self.obj = self.objTry
        self.control = self.controlTry
        self.state = self.stateTry
        self._control_version += 1

    def _control_key(self):
        return (id(self.control),) + tuple(v.data_ptr() for v in self.control.values() if isinstance(v, torch.Tensor))

    def setUpdate(self, update):
        lt = self._last_trial
        if (lt is not None and lt[0] is update[0] and lt[1] == float(update[1]) and lt[2] == self._control_version
                and lt[5] == self._control_key()):
            return lt[3], lt[4]
        control = Control()
        for k, v in update[0].items():
            if v is not None and self.control.get(k) is not None:
                control[k] = self.control[k] - update[1] * v
        _, st = self.objectiveFunDef(control, withTrajectory=True)
        return control, st

    def dotProduct_device(self, g1, g2):
        """g1.g2 over the controls as an FP64 device scalar (no host synchronisation)."""
        tot = None
        for k, v in g1.items():
            if v is None or g2.get(k) is None:
                continue
            t = torch.dot(v.reshape(-1), g2[k].reshape(-1))
            tot = t if tot is None else tot + t
        return tot if tot is not None else torch.zeros((), dtype=torch.float64, device=self.x0.device)

    # Controls of at most this many doubles take the L-BFGS direction from one library call (one CTA runs the whole
    # two-loop recursion; at the coarse levels of a warm start the recursion from the host -- ~4 small kernels and
    # Python calls per stored pair -- costs more than the shooting); larger ones run it from the host, whose kernels
    # spread over the GPU.
    LBFGS_FUSED_MAX = 1 << 16

    # Expected decrease of the objective along the first gradient step, as a fraction of the objective, set by a
    # warm start (None: the optimiser's own first step, 1 / |gradient|, as in the reference).
    first_step_gap = None

    def initial_step(self, obj, grd2):
        """The optimiser's first step along -gradient after a warm start: the minimiser t = 2 D / |g|^2 of the
        quadratic model phi(t) = f0 - |g|^2 t + h t^2 / 2 whose minimum lies D = first_step_gap * f0 below f0
        (the initial-step rule 2 (f_k - f_k-1) / phi'(0) of Nocedal & Wright, section 3.5, with the expected
        decrease in place of the previous one). Near an optimum a unit step (1 / |g|) overshoots by orders of
        magnitude and the line search shrinks it one objective evaluation at a time; any D within 10x of the
        true decrease passes in one or two. Used once; None leaves the optimiser's rule."""
        gap, self.first_step_gap = self.first_step_gap, None
        if gap is None or not (grd2 > 0) or not np.isfinite(obj) or obj <= 0:
            return None
        return 2.0 * gap * obj / (self.gradCoeff * grd2)

    def lbfgs_direction(self, grd, history):
        """The optimiser's two-loop recursion (base/bfgs.py:183-198) for gradient `grd` and the stored pairs
        `history` ([s_k, y_k], oldest first) in one call of lddmm_lbfgs_direction, or None when the controls do not
        fit it (the optimiser then runs the recursion itself)."""
        k = self.control_key
        g = grd.get(k)
        m = len(history)
        if g is None or m < 1 or m > nat.LBFGS_MAX_PAIRS or g.numel() > self.LBFGS_FUSED_MAX:
            return None
        if any(v is not None for kk, v in grd.items() if kk != k):
            return None
        S = [h[0].get(k) for h in history]
        Y = [h[1].get(k) for h in history]
        for t in S + Y:
            if t is None or t.dtype != torch.float64 or not t.is_cuda or not t.is_contiguous() or t.numel() != g.numel():
                return None
        g = g.contiguous()
        q = torch.empty_like(g)
        sp = (ctypes.c_void_p * m)(*[t.data_ptr() for t in S])
        yp = (ctypes.c_void_p * m)(*[t.data_ptr() for t in Y])
        nat.check(nat.lib().lddmm_lbfgs_direction(ctypes.cast(sp, ctypes.c_void_p), ctypes.cast(yp, ctypes.c_void_p),
                                                  m, nat.ptr(g), g.numel(), nat.ptr(q), nat.stream_ptr()),
                  'lbfgs_direction')
        return Control({k: q})

    def dotProduct_euclidean(self, g1, g2):
        vals = [self.dotProduct_device(g1, gr) for gr in g2]
        return torch.stack(vals).tolist()

    dotProduct = dotProduct_euclidean

    def addProd(self, dir1, dir2, beta):
        return Control({k: dir1[k] + beta * dir2[k] for k in dir1 if dir1[k] is not None and dir2.get(k) is not None})

    def prod(self, dir1, beta):
        return Control({k: beta * v for k, v in dir1.items() if v is not None})

    def copyDir(self, dir0):
        return Control({k: (v.clone() if isinstance(v, torch.Tensor) else deepcopy(v)) for k, v in dir0.items()})

    def endOfIteration(self, endP=False):
        self.iter += 1
        self.history.append(self.obj)
        self.times.append(time.perf_counter())
        if self.pkBuffer > 50:
            self.resetPK()
        else:
            self.pkBuffer += 1
        target = self.options['targetObjective']
        if target is not None and self.obj is not None and self.obj <= target and not endP:
            raise TargetReached()

    def endOfProcedure(self):
        self.endOfIteration(endP=True)

    def endOptim(self):
        self.fvDef.updateVertices(self.state['xt'][-1].cpu().numpy())

    def saveHdf5(self, fileName):
        """The result record of the reference's saveHdf5 (base/surfaceMatching.py:1506-1555) as an .npz archive:
        the HDF5 group path of each dataset is its key ('LDDMM Results/parameters/Time steps', ...). Written to
        `fileName` with its extension replaced by .npz (h5py is not available); returns that path."""
        import os
        o = self.options
        K, Kd = o['KparDiff'], o['KparDist']
        ctrl = self.control[self.control_key]
        rec = {'parameters/Time steps': self.Tsize,
               'parameters/Deformation Kernel type': K.name,
               'parameters/Deformation Kernel width': np.asarray(K.sigma),
               'parameters/Deformation Kernel order': K.order,
               'parameters/Spatial Varifold Kernel type': Kd.name,
               'parameters/Spatial Varifold width': np.asarray(Kd.sigma),
               'parameters/Spatial Varifold order': Kd.order,
               'template/vertices': self.fv0.vertices, 'template/faces': self.fv0.faces,
               'target/vertices': self.fv1.vertices, 'target/faces': self.fv1.faces,
               'variables/alpha': ctrl.cpu().numpy(), 'variables/affine': 'None'}
        st = self.solveStateEquation(withJacobian=True)
        xt = st['xt']
        self.fvDef.updateVertices(xt[-1].cpu().numpy())
        rec['deformedTemplate/vertices'] = self.fvDef.vertices
        av0 = self.fv0.computeVertexArea()[0]
        rec['descriptors/Jacobian'] = st['Jt'][-1].cpu().numpy()
        rec['descriptors/Surface Jacobian'] = self.fvDef.computeVertexArea()[0] / av0
        rec['descriptors/Displacement'] = (xt[-1] - xt[0]).cpu().numpy()
        path = os.path.splitext(fileName)[0] + '.npz'
        np.savez(path, **{'LDDMM Results/' + k: np.asarray(v) for k, v in rec.items()})
        return path

    def optimizeMatching(self):
        ws = self.options.get('warmStart')
        if ws is not None and not getattr(self, '_warm_started', False):
            # learned / coarse-to-fine warm start (SecondOrderSurfaceMatching): {'model': MomentumProposal or None,
            # 'coarse': [(faces, vertices), ...] coarsest first, optional 'rtol' and 'first_step_gap'}; the record
            # is kept in self.warmStartRecord
            if self.control_key != 'a0':
                raise NotImplementedError('options["warmStart"] applies to SecondOrderSurfaceMatching')
            from .learnedProposal import multilevel_warm_start, warm_start
            if ws.get('coarse'):
                self.warmStartRecord = multilevel_warm_start(self, ws.get('model'), ws['coarse'],
                                                             rtol=ws.get('rtol', 1e-4),
                                                             first_step_gap=ws.get('first_step_gap', 1e-3))
            elif ws.get('model') is not None:
                self.warmStartRecord = warm_start(self, ws['model'], scales=ws.get('scales', (0.5, 0.75, 1.0)))
            self._warm_started = True
        grd = self.getGradient(self.gradCoeff)
        [grd2] = self.dotProduct_euclidean(grd, [grd])
        if self.gradEps < 0:
            self.gradEps = max(1e-5, np.sqrt(grd2) / 10000)
        self.epsMax = 5.
        logging.info(f'gradient tolerance {self.gradEps:.4g}')
        self.reached_target = False
        try:
            _bfgs.bfgs(self, verb=self.options['verb'], maxIter=self.options['maxIter'],
                       TestGradient=self.options['testGradient'], epsInit=self.options['epsInit'],
                       Wolfe=self.options['Wolfe'], lineSearch=self.options['lineSearch'], memory=50)
        except TargetReached:
            self.reached_target = True
            self.endOptim()
        return self.control


class SurfaceMatching(_DeviceMatching):
    """First-order LDDMM surface matching (base/surfaceMatching.py:75)."""
    control_key = 'at'

    def initialize_variables(self):
        self.control['at'] = torch.zeros((self.Tsize, self.npt, 3), dtype=torch.float64, device=self.x0.device)
        self.control['Afft'] = None
        self.state['xt'] = self.x0.unsqueeze(0).repeat(self.Tsize + 1, 1, 1)

    def objectiveFunDef(self, control, var=None, withTrajectory=True, withJacobian=False):
        """sum_t regWeight dt a_t.K(x_t)a_t with the trajectory (base/surfaceMatching.py:468-565)."""
        e = torch.zeros(1, dtype=torch.float64, device=self.x0.device)
        xt = evol.shoot_first_order(self.x0, control['at'], self.options['KparDiff'],
                                    regweight=self.options['regWeight'], energy=e, origin=self.origin)
        st = State(xt=xt)
        return (e[0], st) if withTrajectory or withJacobian else e[0]

    def _gradient(self, coeff=1.0, update=None):
        """(base/surfaceMatching.py:1040-1105, euclidean gradient K(x_t)(2 w a_t - p_{t+1}) / (coeff T))."""
        if update is None:
            control, st = self.control, self.state
        else:
            control, st = self.setUpdate(update)
        px1 = -self.endPointGradient(st['xt'][-1])
        _, dat = evol.first_order_gradient(st['xt'], control['at'], px1, self.options['KparDiff'],
                                           self.options['regWeight'], euclidean=self.euclideanGradient,
                                           origin=self.origin)
        grd = Control()
        grd['at'] = dat / (coeff * self.Tsize)
        return grd

    def randomDir(self):
        return Control(at=torch.randn((self.Tsize, self.npt, 3), dtype=torch.float64, device=self.x0.device))

    def solveStateEquation(self, control=None, withJacobian=False):
        """Trajectory (and log-Jacobian) of the control (base/surfaceMatching.py:116, landmarkDirectEvolutionEuler)."""
        control = self.control if control is None else control
        return evol.landmarkDirectEvolutionEuler(self.x0, control['at'], self.options['KparDiff'],
                                                 options={'withJacobian': withJacobian})


class SecondOrderSurfaceMatching(_DeviceMatching):
    """Geodesic-shooting surface matching (base/secondOrderSurfaceMatching.py:41,
    base/secondOrderPointSetMatching.py:45-494).

    options['processGroup'] (a torch.distributed group, or True for the default group; one process per GPU, every
    rank given the same surfaces and options) shards the target rows of every shooting step, every adjoint step and
    the kinetic term K(x0)a0 over the ranks (base/distributed.py): one all-gather of the new rows per step, an FP64
    all-reduce of the kinetic energy. The data term is evaluated on every rank (it is 10-20% of an iteration), so
    every rank holds the same objective, gradient and BFGS state and takes the same decisions."""
    control_key = 'a0'

    def _sharding(self):
        pg = self.options.get('processGroup')
        if pg is None or pg is False:
            return None
        from . import distributed as dd
        group = None if pg is True else pg
        K = self.options['KparDiff']
        key = (id(group), K.pk_dtype)
        if getattr(self, '_shard_key', None) != key:
            self._shard = (dd, group, dd.library_step_rows(K, self.origin), dd.library_adjoint_rows(K, self.origin),
                           dd.library_k_rows(K, self.origin), dd.RowGather(self.npt, 3, torch.float64, self.x0.device,
                                                                           group))
            self._shard_key = key
        return self._shard

    def initialize_variables(self):
        a0 = self.options['initialMomentum']
        self._zero_start = None
        if a0 is None:
            # zero momentum: the geodesic stays at x0 with zero momentum (what shooting it gives, exactly), so the
            # trajectory is written instead of shot; objectiveFunDef recognises this control by identity
            self.control['a0'] = torch.zeros((self.npt, 3), dtype=torch.float64, device=self.x0.device)
            T = int(np.round(1.0 / self.options['timeStep']))
            xt = self.x0.unsqueeze(0).repeat(T + 1, 1, 1)
            at = torch.zeros((T + 1, self.npt, 3), dtype=torch.float64, device=self.x0.device)
            self._zero_start = (self.control['a0'], State(xt=xt, at=at))
        else:
            self.control['a0'] = nat.as_device(a0).clone()
            xt, at = evol.shoot_second_order(self.x0, self.control['a0'], self.options['KparDiff'],
                                             self.options['timeStep'], origin=self.origin)
        self.control['Afft'] = None
        self.state = State(xt=xt, at=at)

    def objectiveFunDef(self, control, var=None, withTrajectory=True, withJacobian=False):
        """0.5 a0.K(x0)a0 with the geodesic trajectory (base/secondOrderPointSetMatching.py:113-148)."""
        K = self.options['KparDiff']
        a0 = control['a0']
        zs = getattr(self, '_zero_start', None)
        if zs is not None and a0 is zs[0]:
            # the untouched zero start: kinetic energy 0 and the constant trajectory
            obj = torch.zeros((), dtype=torch.float64, device=self.x0.device)
            return (obj, zs[1]) if withTrajectory or withJacobian else obj
        sh = self._sharding()
        if sh is not None:
            dd, group, step_rows, _, k_rows, gather = sh
            xt, at = dd.sharded_second_order_shoot(self.x0, a0, self.options['timeStep'], step_rows, group, gather)
            obj, _ = dd.sharded_kinetic(self.x0, a0, k_rows, group, gather)
            st = State(xt=xt, at=at)
            return (obj, st) if withTrajectory or withJacobian else obj
        xt, at = evol.shoot_second_order(self.x0, a0, K, self.options['timeStep'], origin=self.origin)
        obj = 0.5 * (a0 * K._apply_k(self.x0, self.x0, a0, float(np.asarray(K.sigma).ravel()[0]), self.origin)).sum() \
            if np.asarray(K.sigma).size == 1 else 0.5 * (a0 * K.applyK(self.x0, a0)).sum()
        st = State(xt=xt, at=at)
        return (obj, st) if withTrajectory or withJacobian else obj

    def _gradient(self, coeff=1.0, update=None):
        """da0 = K(x0)a0 - pa_0 after the adjoint sweep (base/secondOrderPointSetMatching.py:379-483)."""
        if update is None:
            control, st = self.control, self.state
        else:
            control, st = self.setUpdate(update)
        px1 = -self.endPointGradient(st['xt'][-1])
        pa1 = torch.zeros_like(px1)
        sh = self._sharding()
        if sh is not None:
            dd, group, _, adjoint_rows, k_rows, gather = sh
            _, pat = dd.sharded_second_order_adjoint(st['xt'], st['at'], px1, pa1, self.options['timeStep'],
                                                     adjoint_rows, group, gather)
            _, ka0 = dd.sharded_kinetic(self.x0, control['a0'], k_rows, group, gather)
            grd = Control()
            grd['a0'] = (ka0 - pat[0]) / coeff
            return grd
        _, _, da0 = evol.second_order_adjoint(st['xt'], st['at'], px1, pa1, self.options['KparDiff'],
                                              self.options['timeStep'], origin=self.origin)
        grd = Control()
        grd['a0'] = da0 / coeff
        return grd

    def randomDir(self):
        return Control(a0=torch.randn((self.npt, 3), dtype=torch.float64, device=self.x0.device))

    def solveStateEquation(self, control=None, withJacobian=False):
        """Geodesic trajectory (and log-Jacobian) of the control (base/secondOrderPointSetMatching.py:100,
        secondOrderEvolution)."""
        control = self.control if control is None else control
        return evol.secondOrderEvolution(self.x0, control['a0'], self.options['KparDiff'], self.options['timeStep'],
                                         options={'withJacobian': withJacobian})
