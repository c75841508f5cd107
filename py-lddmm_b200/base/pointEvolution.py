"""Drop-in landmark shooting and adjoint (reference: base/pointEvolution.py:88-618) on the B200.

Single-width Gaussian kernels go through the fused trajectory entry points of the library (one exp per pair
shared by every sum of a time step, FP64 state accumulation across steps); multi-width kernels compose the
per-operator `Kernel` methods step by step (still on the device). Affine components are not implemented.
Inputs are numpy or torch; outputs have the type of `x0`.
"""
import numpy as np
import torch

from . import _native as nat


def _is_np(v):
    return not isinstance(v, torch.Tensor)


def _ret(t, like_np):
    if t is None:
        return None
    return t.cpu().numpy() if like_np else t


def _no_affine(affine):
    if affine is not None and len(affine) > 0 and affine[0] is not None and len(affine[0]) > 0:
        raise NotImplementedError('lddmm_b200 does not implement affine components in shooting')


def _single_sigma(K):
    K._check()
    s = np.asarray(K.sigma, dtype=float).ravel()
    return float(s[0]) if s.size == 1 else None


def shoot_first_order(X0, AT, K, regweight=1.0, energy=None, origin=None):
    """Device-level: xt (T+1,N,3) and optional kinetic energy regweight*dt*sum_t a_t.K(x_t)a_t (1-elem tensor)."""
    T, N = AT.shape[0], AT.shape[1]
    sig = _single_sigma(K)
    xt = torch.empty((T + 1, N, 3), dtype=torch.float64, device=X0.device)
    if sig is None:
        xt[0] = X0
        e = torch.zeros(1, dtype=torch.float64, device=X0.device)
        for t in range(T):
            ka = K.applyK(xt[t], AT[t])
            xt[t + 1] = xt[t] + ka / T
            e += regweight / T * (AT[t] * ka).sum()
        if energy is not None:
            energy.copy_(e)
        return xt
    ws, wsb = nat.workspace(N, N, K.precision)
    o = nat.origin_arg(origin if origin is not None else nat.centroid(X0))
    nat.check(nat.lib().lddmm_first_order_shoot(nat.ptr(X0), nat.ptr(AT), N, T, sig, K.code, float(regweight), o,
                                                nat.ptr(xt), nat.ptr(energy), K.precision, ws, wsb, nat.stream_ptr()),
              'first_order_shoot')
    return xt


def first_order_gradient(XT, AT, PX1, K, regweight, euclidean=False, origin=None):
    """Device-level adjoint: returns (pxt (T+1,N,3), dat (T,N,3)) with dat = 2w a - p (or K(x)(2w a - p))."""
    T, N = AT.shape[0], AT.shape[1]
    sig = _single_sigma(K)
    pxt = torch.empty((T + 1, N, 3), dtype=torch.float64, device=XT.device)
    dat = torch.empty((T, N, 3), dtype=torch.float64, device=XT.device)
    if sig is None:
        pxt[T] = PX1
        for t in range(T - 1, -1, -1):
            px = pxt[t + 1]
            pxt[t] = px + K.applyDiffKT(XT[t], px, AT[t], regweight=regweight, lddmm=True) / T
            g = 2 * regweight * AT[t] - px
            dat[t] = K.applyK(XT[t], g) if euclidean else g
        return pxt, dat
    ws, wsb = nat.workspace(N, N, K.precision)
    o = nat.origin_arg(origin if origin is not None else nat.centroid(XT[0]))
    nat.check(nat.lib().lddmm_first_order_gradient(nat.ptr(XT), nat.ptr(AT), N, T, sig, K.code, float(regweight),
                                                   nat.ptr(PX1.contiguous()), int(bool(euclidean)), o, nat.ptr(pxt),
                                                   nat.ptr(dat), K.precision, ws, wsb, nat.stream_ptr()),
              'first_order_gradient')
    return pxt, dat


def shoot_second_order(X0, A0, K, timeStep, origin=None):
    """Device-level geodesic shooting: (xt, at), each (T+1,N,3), T = round(1/timeStep), step size timeStep."""
    T = int(np.round(1.0 / timeStep))
    N = X0.shape[0]
    sig = _single_sigma(K)
    xt = torch.empty((T + 1, N, 3), dtype=torch.float64, device=X0.device)
    at = torch.empty((T + 1, N, 3), dtype=torch.float64, device=X0.device)
    if sig is None:
        xt[0], at[0] = X0, A0
        for k in range(T):
            xt[k + 1] = xt[k] + timeStep * K.applyK(xt[k], at[k])
            at[k + 1] = at[k] - timeStep * K.applyDiffKT(xt[k], at[k], at[k])
        return xt, at
    ws, wsb = nat.workspace(N, N, K.precision)
    o = nat.origin_arg(origin if origin is not None else nat.centroid(X0))
    nat.check(nat.lib().lddmm_second_order_shoot(nat.ptr(X0), nat.ptr(A0), N, T, sig, K.code, float(timeStep), o,
                                                 nat.ptr(xt), nat.ptr(at), K.precision, ws, wsb, nat.stream_ptr()),
              'second_order_shoot')
    return xt, at


def second_order_adjoint(XT, AT, PX1, PA1, K, timeStep, origin=None, with_da0=True):
    """Device-level adjoint sweep: (pxt, pat, da0) with da0 = K(x0) a0 - pa_0."""
    T = XT.shape[0] - 1
    N = XT.shape[1]
    sig = _single_sigma(K)
    pxt = torch.empty_like(XT)
    pat = torch.empty_like(XT)
    da0 = torch.empty((N, 3), dtype=torch.float64, device=XT.device) if with_da0 else None
    if sig is None:
        pxt[T], pat[T] = PX1, PA1
        for t in range(T - 1, -1, -1):
            px, pa, x, a = pxt[t + 1], pat[t + 1], XT[t], AT[t]
            zpx = K.applyDiffKT(x, px, a, sym=True) - K.applyDDiffK11and12(x, a, a, pa)
            zpa = K.applyK(x, px) - K.applyDiffK1and2(x, pa, a)
            pxt[t] = px + timeStep * zpx
            pat[t] = pa + timeStep * zpa
        if with_da0:
            da0.copy_(K.applyK(XT[0], AT[0]) - pat[0])
        return pxt, pat, da0
    ws, wsb = nat.workspace(N, N, K.precision)
    o = nat.origin_arg(origin if origin is not None else nat.centroid(XT[0]))
    nat.check(nat.lib().lddmm_second_order_gradient(nat.ptr(XT), nat.ptr(AT), N, T, sig, K.code, float(timeStep),
                                                    nat.ptr(PX1.contiguous()), nat.ptr(PA1.contiguous()), o,
                                                    nat.ptr(pxt), nat.ptr(pat), nat.ptr(da0), K.precision, ws, wsb,
                                                    nat.stream_ptr()), 'second_order_gradient')
    return pxt, pat, da0


# ---------------------------------------------------------------------------------------------------------------
# Reference-signature wrappers
# ---------------------------------------------------------------------------------------------------------------
def landmarkDirectEvolutionEuler(x0, at, KparDiff, affine=None, options=None):
    """x_{t+1} = x_t + dt K(x_t) a_t (base/pointEvolution.py:88-164); returns dict(xt, Jt, yt, nt)."""
    _no_affine(affine)
    opts = {'withJacobian': False, 'withNormals': None, 'withPointSet': None}
    if options is not None:
        opts.update(options)
    like_np = _is_np(x0)
    X0, AT = nat.as_device(x0), nat.as_device(at)
    T, N = AT.shape[0], AT.shape[1]
    xt = shoot_first_order(X0, AT, KparDiff)
    dt = 1.0 / T
    Jt = yt = nt = None
    if opts['withPointSet'] is not None:
        Y0 = nat.as_device(opts['withPointSet'])
        yt = torch.empty((T + 1,) + tuple(Y0.shape), dtype=torch.float64, device=X0.device)
        yt[0] = Y0
        for t in range(T):
            yt[t + 1] = yt[t] + dt * KparDiff.applyK(xt[t], AT[t], firstVar=yt[t])
    if opts['withJacobian']:
        M = yt.shape[1] if yt is not None else N
        Jt = torch.zeros((T + 1, M, 1), dtype=torch.float64, device=X0.device)
        for t in range(T):
            fv = yt[t] if yt is not None else None
            Jt[t + 1] = Jt[t] + dt * KparDiff.applyDivergence(xt[t], AT[t], firstVar=fv)
    if opts['withNormals'] is not None:
        N0 = nat.as_device(opts['withNormals'])
        nt = torch.empty((T + 1, N, 3), dtype=torch.float64, device=X0.device)
        nt[0] = N0
        for t in range(T):
            nt[t + 1] = nt[t] - dt * KparDiff.applyDiffKT(xt[t], nt[t], AT[t])
    return {'xt': _ret(xt, like_np), 'Jt': _ret(Jt, like_np), 'yt': _ret(yt, like_np), 'nt': _ret(nt, like_np)}


def landmarkHamiltonianCovector(x0, at, px1, Kpardiff, regweight, affine=None, extraTerm=None):
    """Backward p_t = p_{t+1} + dt DK^T_lddmm (base/pointEvolution.py:167-201); returns (pxt, xt)."""
    _no_affine(affine)
    if extraTerm is not None:
        raise NotImplementedError('extraTerm is not implemented')
    like_np = _is_np(x0)
    X0, AT, PX1 = nat.as_device(x0), nat.as_device(at), nat.as_device(px1)
    xt = shoot_first_order(X0, AT, Kpardiff)
    pxt, _ = first_order_gradient(xt, AT, PX1, Kpardiff, regweight)
    return _ret(pxt, like_np), _ret(xt, like_np)


def landmarkHamiltonianGradient(x0, at, px1, KparDiff, regweight, getCovector=False, affine=None, extraTerm=None):
    """dat_t = 2 w a_t - p_{t+1} (base/pointEvolution.py:205-236); returns (dat, xt[, pxt])."""
    _no_affine(affine)
    if extraTerm is not None:
        raise NotImplementedError('extraTerm is not implemented')
    like_np = _is_np(x0)
    X0, AT, PX1 = nat.as_device(x0), nat.as_device(at), nat.as_device(px1)
    xt = shoot_first_order(X0, AT, KparDiff)
    pxt, dat = first_order_gradient(xt, AT, PX1, KparDiff, regweight)
    if getCovector:
        return _ret(dat, like_np), _ret(xt, like_np), _ret(pxt, like_np)
    return _ret(dat, like_np), _ret(xt, like_np)


def secondOrderEvolution(x0, a0, KparDiff, timeStep, withSpline=None, affine=None, options=None):
    """Geodesic shooting (base/pointEvolution.py:385-472); returns dict(xt, at, Jt, yt)."""
    _no_affine(affine)
    if withSpline is not None:
        raise NotImplementedError('withSpline is not implemented')
    opts = {'withJacobian': False, 'withNormals': None, 'withPointSet': None}
    if options is not None:
        opts.update(options)
    like_np = _is_np(x0)
    X0, A0 = nat.as_device(x0), nat.as_device(a0)
    xt, at = shoot_second_order(X0, A0, KparDiff, timeStep)
    T = xt.shape[0] - 1
    Jt = zt = None
    if opts['withPointSet'] is not None:
        Z0 = nat.as_device(opts['withPointSet'])
        zt = torch.empty((T + 1,) + tuple(Z0.shape), dtype=torch.float64, device=X0.device)
        zt[0] = Z0
        for k in range(T):
            zt[k + 1] = zt[k] + timeStep * KparDiff.applyK(xt[k], at[k], firstVar=zt[k])
    if opts['withJacobian']:
        M = zt.shape[1] if zt is not None else X0.shape[0]
        Jt = torch.zeros((T + 1, M, 1), dtype=torch.float64, device=X0.device)
        for k in range(T):
            fv = zt[k] if zt is not None else None
            Jt[k + 1] = Jt[k] + timeStep * KparDiff.applyDivergence(xt[k], at[k], firstVar=fv)
    return {'xt': _ret(xt, like_np), 'at': _ret(at, like_np), 'Jt': _ret(Jt, like_np), 'yt': _ret(zt, like_np)}


def landmarkEPDiff(T, x0, a0, KparDiff, affine=None, withJacobian=False, withNormals=None, withPointSet=None):
    """Geodesic (EPDiff) shooting over T steps of 1/T (base/pointEvolution.py:320-382): xt (T+1,N,3) and at (T,N,3)
    from the fused shooting kernels; with a point set, normals or the Jacobian requested, the list
    [xt, at, (yt), (nt), (Jt)] in the reference's order (yt carried by K(x_t, .) a_t, nt by -DK^T(x_t; n_t, a_t),
    Jt by the divergence of K(x_t, .) a_t at the points x_t)."""
    _no_affine(affine)
    like_np = _is_np(x0)
    X0, A0 = nat.as_device(x0), nat.as_device(a0)
    T = int(T)
    dt = 1.0 / T
    xt, at_all = shoot_second_order(X0, A0, KparDiff, dt)
    at = at_all[:T]
    out = [_ret(xt, like_np), _ret(at.contiguous(), like_np)]
    if withPointSet is not None:
        Y0 = nat.as_device(withPointSet)
        yt = torch.empty((T + 1,) + tuple(Y0.shape), dtype=torch.float64, device=X0.device)
        yt[0] = Y0
        for k in range(T):
            yt[k + 1] = yt[k] + dt * KparDiff.applyK(xt[k], at[k], firstVar=yt[k])
        out.append(_ret(yt, like_np))
    if withNormals is not None:
        N0 = nat.as_device(withNormals)
        nt = torch.empty((T + 1,) + tuple(N0.shape), dtype=torch.float64, device=X0.device)
        nt[0] = N0
        for k in range(T):
            nt[k + 1] = nt[k] - dt * KparDiff.applyDiffKT(xt[k], nt[k], at[k])
        out.append(_ret(nt, like_np))
    if withJacobian:
        Jt = torch.zeros((T + 1, X0.shape[0], 1), dtype=torch.float64, device=X0.device)
        for k in range(T):
            Jt[k + 1] = Jt[k] + dt * KparDiff.applyDivergence(xt[k], at[k])
        out.append(_ret(Jt, like_np))
    return (out[0], out[1]) if len(out) == 2 else out


def secondOrderHamiltonian(x, a, px, pa, KparDiff, withSpline=None, affine=None):
    """H = px.K(x)a - pa.DK^T(x; a, a) (base/pointEvolution.py:475-486)."""
    _no_affine(affine)
    like_np = _is_np(x)
    X, A, PX, PA = (nat.as_device(v) for v in (x, a, px, pa))
    H = (PX * KparDiff.applyK(X, A)).sum() - (PA * KparDiff.applyDiffKT(X, A, A)).sum()
    if withSpline is not None:
        S = nat.as_device(withSpline)
        H = H + (PA * S).sum() - (S ** 2).sum() / 2
    return float(H) if like_np else H


def secondOrderCovector(x0, a0, px1, pa1, KparDiff, timeStep, withSpline=None, affine=None, isjump=None,
                        forwardState=None):
    """Adjoint sweep (base/pointEvolution.py:489-552); returns (pxt, pat, xt, at)."""
    _no_affine(affine)
    if withSpline is not None or (isjump is not None and np.any(isjump)):
        raise NotImplementedError('splines and multi-target jumps are not implemented')
    like_np = _is_np(x0)
    if isinstance(px1, (list, tuple)):
        if len(px1) != 1:
            raise NotImplementedError('multiple targets are not implemented')
        px1, pa1 = px1[0], pa1[0]
    X0, A0, PX1, PA1 = nat.as_device(x0), nat.as_device(a0), nat.as_device(px1), nat.as_device(pa1)
    if forwardState is None:
        xt, at = shoot_second_order(X0, A0, KparDiff, timeStep)
    else:
        xt, at = nat.as_device(forwardState[0]), nat.as_device(forwardState[1])
    pxt, pat, _ = second_order_adjoint(xt, at, PX1, PA1, KparDiff, timeStep, with_da0=False)
    return _ret(pxt, like_np), _ret(pat, like_np), _ret(xt, like_np), _ret(at, like_np)


def secondOrderGradient(x0, a0, px1, pa1, KparDiff, timeStep, isjump=None, withSpline=None, affine=None,
                        controlWeight=1.0):
    """Gradient of geodesic shooting (base/pointEvolution.py:555-618): dict(da0, drhot, xt, at, dA, db, pxt, pat)."""
    _no_affine(affine)
    if withSpline is not None:
        raise NotImplementedError('withSpline is not implemented')
    like_np = _is_np(x0)
    X0, A0, PX1, PA1 = nat.as_device(x0), nat.as_device(a0), nat.as_device(px1), nat.as_device(pa1)
    xt, at = shoot_second_order(X0, A0, KparDiff, timeStep)
    pxt, pat, da0 = second_order_adjoint(xt, at, PX1, PA1, KparDiff, timeStep)
    return {'da0': _ret(da0, like_np), 'drhot': None, 'xt': _ret(xt, like_np), 'at': _ret(at, like_np), 'dA': None,
            'db': None, 'pxt': _ret(pxt, like_np), 'pat': _ret(pat, like_np)}
