"""Host-side logic that needs no GPU: the conjugate-gradient solver, and the optimiser's failure handling.

Failure handling follows the reference: a NaN objective at a trial point is reported as 1e500 so that the line
search rejects the step (base/surfaceMatching.py:666-668); a failed line search sets `reset`, and the next iteration
switches the kernel sums to float64 (base/surfaceMatching.py:1340-1345) and restarts BFGS from a plain gradient
step; a second failure right after a restart stops the optimiser (base/bfgs.py:241-258). The failures are made on
the host: a test double of the matching class whose objective is a small quadratic on CPU tensors, with a NaN or
a wrong-sign gradient planted in it. Nothing here runs a kernel.
"""
import numpy as np
import pytest
import torch

from base import _native as nat
from base import bfgs as bfgs_mod
from base.conjugateGradient import linearcg
from base.kernelFunctions import Kernel
from base.linesearch import line_search_weak_wolfe
from base.surfaceMatching import Control, State, _DeviceMatching


def test_linearcg_matches_dense_solve():
    rng = np.random.default_rng(3)
    x = rng.normal(size=(60, 3))
    d2 = ((x[:, None, :] - x[None, :, :]) ** 2).sum(-1)
    A = np.exp(-d2 / (2 * 0.8 ** 2)) + 0.05 * np.eye(60)     # Gaussian kernel matrix + ridge: SPD
    b = rng.normal(size=(60, 3))
    got = linearcg(lambda v: A @ v, b, iterMax=400, tol=1e-12)
    ref = np.linalg.solve(A, b)
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 1e-9
    # warm start and the torch-tensor path
    got_t = linearcg(lambda v: torch.from_numpy(A) @ v, torch.from_numpy(b), iterMax=400,
                     x0=torch.zeros(60, 3, dtype=torch.float64), tol=1e-12)
    assert np.linalg.norm(got_t.numpy() - ref) / np.linalg.norm(ref) < 1e-9
    # zero right-hand side: the zero vector, no operator call needed
    assert np.all(linearcg(lambda v: A @ v, np.zeros((60, 3))) == 0)


class _FakeData:
    def __init__(self):
        self.precision = nat.FP32C

    def norm0(self):
        return 0.0


class QuadraticMatching(_DeviceMatching):
    """The matching protocol of _DeviceMatching on a CPU quadratic 0.5 |a - c|^2 (no kernels). `nan_above`
    makes the objective NaN for trial controls farther than that from the origin; `flip_gradient` returns the
    gradient with the wrong sign, so every line search fails."""

    def __init__(self, n=8, nan_above=None, flip_gradient=False):
        self.options = self.getDefaultOptions()
        self.options.update(KparDiff=Kernel(name='gauss', sigma=0.5), KparDist=Kernel(name='gauss', sigma=0.3),
                            verb=False)
        self.Kdiff_dtype = 'float32'
        self.data = _FakeData()
        self.resetPK('float32')
        self.x0 = torch.zeros((n, 3), dtype=torch.float64)
        self.npt, self.Tsize, self.sigma2 = n, 1, 1.0
        self.euclideanGradient, self.gradCoeff, self.gradEps, self.burnIn = True, 1.0, 1e-12, 0
        self.obj = self.objTry = None
        self.reset = False
        self.iter = self.pkBuffer = 0
        self.history, self.times = [], []
        self._last_trial = self._grad_cache = None
        self._control_version = 0
        self.c = torch.linspace(-1.0, 1.0, 3 * n, dtype=torch.float64).reshape(n, 3)
        self.control = Control(a0=torch.zeros((n, 3), dtype=torch.float64))
        self.controlTry = Control()
        self.state = State(xt=torch.zeros((2, n, 3), dtype=torch.float64))
        self.stateTry = None
        self.nan_above = nan_above
        self.flip = flip_gradient
        self.evaluations = 0
        self.precisions_seen = []

    def objectiveFunDef(self, control, var=None, withTrajectory=True, withJacobian=False):
        self.evaluations += 1
        self.precisions_seen.append(self.options['KparDiff'].pk_dtype)
        a = control['a0']
        obj = 0.5 * float(((a - self.c) ** 2).sum())
        if self.nan_above is not None and float(a.norm()) > self.nan_above:
            obj = float('nan')
        return obj, State(xt=torch.zeros((2, self.npt, 3), dtype=torch.float64))

    def dataTerm(self, xdef):
        return 0.0

    def endOptim(self):
        pass

    def _gradient(self, coeff=1.0, update=None):
        a = self.control['a0'] if update is None else self.control['a0'] - update[1] * update[0]['a0']
        g = a - self.c
        return Control(a0=(-g if self.flip else g) / coeff)


def test_nan_trial_objective_is_rejected():
    m = QuadraticMatching(nan_above=0.5)
    m.objectiveFun()
    base_obj = m.obj
    g = m.getGradient(1.0)
    # a long step lands beyond the NaN radius: reported as 1e500 and the trial control is not kept
    f = m.updateTry(g, 10.0, base_obj)
    assert f == 1e500
    assert m.objTry is None and not m.controlTry
    # the line search backs off from the NaN region and accepts a finite, decreasing step
    t, fc, gc, f_star, f0, _ = line_search_weak_wolfe(m, g, gfk=g, old_fval=base_obj, t_init=10.0, maxiter=10)
    assert t is not None and 0 < t < 10.0
    assert np.isfinite(f_star) and f_star < base_obj
    assert fc >= 2


def test_failed_line_search_resets_to_float64_then_stops():
    m = QuadraticMatching(flip_gradient=True)
    assert m.options['KparDiff'].pk_dtype == 'float32' and m.data.precision == nat.FP32C
    bfgs_mod.bfgs(m, verb=False, maxIter=20, epsInit=1.0, Wolfe=True, lineSearch='Weak_Wolfe', memory=5)
    # first failure: reset; the next iteration runs in float64; the second failure stops the optimiser
    assert m.options['KparDiff'].pk_dtype == 'float64'
    assert m.options['KparDist'].pk_dtype == 'float64'
    assert m.data.precision == nat.FP64
    assert m.converged is False
    assert 'float32' in m.precisions_seen and m.precisions_seen[-1] == 'float64'
    # two searches of at most 100 trial steps each, plus the objective re-evaluated at the restart
    assert m.evaluations <= 2 * 101 + 2
    assert m.iter <= 3
    # the control never moved: every trial was uphill
    assert float(m.control['a0'].abs().max()) == 0.0


def test_working_gradient_converges():
    m = QuadraticMatching()
    bfgs_mod.bfgs(m, verb=False, maxIter=50, epsInit=1.0, Wolfe=True, lineSearch='Weak_Wolfe', memory=5)
    assert float((m.control['a0'] - m.c).abs().max()) < 1e-6
    assert m.options['KparDiff'].pk_dtype == 'float32'


class _IllConditioned(QuadraticMatching):
    """0.5 (a - c)^T D (a - c) with D spread over two decades: BFGS needs several iterations and keeps pairs."""

    def __init__(self, hook=None):
        super().__init__()
        self.D = torch.logspace(-1, 1, 3 * self.npt, dtype=torch.float64).reshape(self.npt, 3)
        self.hook = hook
        self.hook_calls = 0

    def objectiveFunDef(self, control, var=None, withTrajectory=True, withJacobian=False):
        self.evaluations += 1
        a = control['a0']
        return 0.5 * float((self.D * (a - self.c) ** 2).sum()), State(xt=torch.zeros((2, self.npt, 3),
                                                                                      dtype=torch.float64))

    def _gradient(self, coeff=1.0, update=None):
        a = self.control['a0'] if update is None else self.control['a0'] - update[1] * update[0]['a0']
        return Control(a0=self.D * (a - self.c) / coeff)

    def lbfgs_direction(self, grd, history):
        self.hook_calls += 1
        return None if self.hook is None else self.hook(grd, history)


def _compact_lbfgs(grd, history):
    """H g by the compact representation of L-BFGS (Byrd, Nocedal and Schnabel 1994) -- mathematically the two-loop
    recursion with H0 = gamma I, gamma = s.y / y.y of the newest pair, computed another way."""
    g = grd['a0'].reshape(-1).numpy()
    S = np.stack([h[0]['a0'].reshape(-1).numpy() for h in history], axis=1)
    Y = np.stack([h[1]['a0'].reshape(-1).numpy() for h in history], axis=1)
    gamma = (S[:, -1] @ Y[:, -1]) / (Y[:, -1] @ Y[:, -1])
    SY = S.T @ Y
    R = np.triu(SY)
    Dm = np.diag(np.diag(SY))
    Rinv = np.linalg.inv(R)
    M = np.block([[Rinv.T @ (Dm + gamma * Y.T @ Y) @ Rinv, -Rinv.T], [-Rinv, np.zeros_like(R)]])
    W = np.concatenate([S, gamma * Y], axis=1)
    q = gamma * g + W @ (M @ (W.T @ g))
    return Control(a0=torch.from_numpy(q.reshape(grd['a0'].shape).copy()))


def test_bfgs_fused_direction_hook():
    """The optimiser's `lbfgs_direction` hook: a hook that returns the direction (here by the compact representation)
    gives the iterates of the two-loop recursion; a hook that returns None falls back to the recursion."""
    runs = {}
    for name, hook in (('recursion', None), ('compact', _compact_lbfgs)):
        m = _IllConditioned(hook=hook)
        bfgs_mod.bfgs(m, verb=False, maxIter=25, epsInit=1.0, Wolfe=True, lineSearch='Weak_Wolfe', memory=5)
        runs[name] = (np.array(m.history), m)
    (h_rec, m_rec), (h_cmp, m_cmp) = runs['recursion'], runs['compact']
    assert m_rec.hook_calls >= 5 and m_cmp.hook_calls == m_rec.hook_calls     # called at every iteration with pairs
    assert h_rec.shape == h_cmp.shape and h_rec.shape[0] >= 6
    assert np.max(np.abs(h_rec - h_cmp)) <= 1e-10 * np.max(np.abs(h_rec))
    assert h_cmp[-1] < 1e-4 * h_cmp[0]


def test_bfgs_initial_step_hook():
    """The first step after a warm start (`first_step_gap`): started near the optimum of the ill-conditioned
    quadratic, the optimiser's own first trial (1 / |g|) overshoots and the line search shrinks it over several
    objective evaluations; with the expected decrease given, the first trial is 2 D / |g|^2 and is accepted at once.
    Without the gap the hook leaves the optimiser's rule (the reference's first step)."""
    trials = {}
    for gap in (None, 'exact'):
        m = _IllConditioned()
        m.control = Control(a0=m.c + 1e-3 * torch.cos(torch.arange(3 * m.npt, dtype=torch.float64)).reshape(m.npt, 3))
        m.obj = None
        f0 = m.objectiveFun()
        g = m.D * (m.control['a0'] - m.c)
        g2 = float((g * g).sum())
        if gap == 'exact':   # the decrease of the exact line minimum along -g: (g.g)^2 / (2 g.D g)
            m.first_step_gap = g2 ** 2 / (2 * float((g * m.D * g).sum())) / f0
        seen = []
        update_try = m.updateTry

        def record(dr, eps, objRef=None, update_try=update_try, seen=seen):
            seen.append(float(eps))
            return update_try(dr, eps, objRef)
        m.updateTry = record
        bfgs_mod.bfgs(m, verb=False, maxIter=1, epsInit=1.0, Wolfe=True, lineSearch='Weak_Wolfe', memory=5)
        trials[gap] = (seen, m.obj, f0, g2)
        assert m.first_step_gap is None                     # used once
    seen, obj, f0, g2 = trials[None]
    assert seen[0] == pytest.approx(1 / np.sqrt(g2)) and len(seen) >= 3 and obj < f0
    seen_h, obj_h, f0_h, _ = trials['exact']
    assert f0_h == f0 and len(seen_h) == 1 and obj_h < f0
    assert seen_h[0] < seen[0] / 10
