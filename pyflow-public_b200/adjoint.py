"""Discrete adjoint of the time step behind ``torch.autograd.Function``.

One forward step is u_{n+1} = P(R(u_n)): R the RK4 (or Euler) predictor with
the reference's stage-4 state u + dt/2 k3 (src/solver/advancer.py:75-113) and
P = I - G L^-1 D the projection of Domain.velCorr (src/data/domain.py:373-402;
rho/dt cancels).  Because D^T = -G on the staggered periodic grid, P^T = P, so
the adjoint projection is the projection itself -- as in the reference's
Domain.adjointStep (src/data/domain.py:409-438).  The predictor is reversed
stage by stage (for RK4 with h = dt/2):

    lam* = P lam
    m4 = J(u4)^T (dt/6 lam*)          m3 = J(u3)^T (dt/3 lam* + h m4)
    m2 = J(u2)^T (dt/3 lam* + h m3)   m1 = J(u1)^T (dt/6 lam* + h m2)
    lam_n = lam* + m1 + m2 + m3 + m4

with J^T from the hand-written kernel pf_rhs_adjoint and the stage states
u2..u4 recomputed from the saved step input (per-step checkpoints, stage
recomputation).  With 'tensor' SFS stresses F held fixed over the step (the
reference evaluates them once per step, src/data/domain.py:353-355), the
adjoint of F is accumulated by pf_sfs_adjoint over the four stages.

The reference's own RK4 adjoint freezes the forward state at the start of the
step (src/solver/adjoint.py:86-88,174-227) and is therefore exact only for
Euler; this one is exact for both.
"""
import ctypes

import torch

from . import _lib as L
from . import ops

_lib = L.lib()
_P = ctypes.c_void_p
_D = ctypes.c_double
_G = ctypes.POINTER(L.Grid)
_lib.pf_rhs_adjoint.argtypes = [_G, _P, _P, _P, _P, _P, _P, _D, _D, _P, _P, _P, _P]
_lib.pf_rhs_adjoint.restype = ctypes.c_int
_lib.pf_sfs_adjoint.argtypes = [_G, _P, _P, _P, _D, _P, _P]
_lib.pf_sfs_adjoint.restype = ctypes.c_int


def rhs_adjoint(state, lam, spacing, mu, rho):
    """J(state)^T lam for the constant-viscosity RHS (pf_rhs_adjoint)."""
    u, v, w = state
    out = tuple(torch.empty_like(u) for _ in range(3))
    g = ops.grid(u.shape, spacing)
    L.check("pf_rhs_adjoint", _lib.pf_rhs_adjoint(
        ctypes.byref(g), ops._p(u), ops._p(v), ops._p(w), ops._p(lam[0]),
        ops._p(lam[1]), ops._p(lam[2]), float(mu), float(rho), ops._p(out[0]),
        ops._p(out[1]), ops._p(out[2]), ops._stream(u)))
    return out


def sfs_adjoint_accumulate(lam, spacing, weight, out):
    """out (6, nx, ny, nz) += weight * adjoint of the tensor SFS stresses."""
    g = ops.grid(lam[0].shape, spacing)
    L.check("pf_sfs_adjoint", _lib.pf_sfs_adjoint(
        ctypes.byref(g), ops._p(lam[0]), ops._p(lam[1]), ops._p(lam[2]),
        float(weight), ops._p(out), ops._stream(lam[0])))


def project(vel, spacing, rho, dt, tol=1e-12, max_it=20000, p=None, DP=None):
    """In-place projection P vel = vel - G L^-1 D vel (FP64 BiCGStab): the
    target-data corrector Domain.TargetDataVelCorr (src/data/domain.py:445-468),
    divergence, pressure solve from DP = 0, vel -= dt/rho grad DP.  The
    reference's solve also adds DP to the pressure it is given (the
    simulation's p): pass ``p`` to get that; ``DP`` receives the solution."""
    u, v, w = vel
    src = ops.div_vel(u, v, w, spacing)
    DP = torch.zeros_like(u) if DP is None else DP.zero_()
    p = torch.zeros_like(u) if p is None else p
    # a field that is already divergence free to the solver's precision (the
    # adjoint of a loss between two projected fields: its divergence is
    # round-off of the field) needs no correction: BiCGStab on a round-off
    # right-hand side only iterates on noise, stagnates at the relative
    # tolerance and can end non-finite
    vmax = max(float(t.abs().max()) for t in vel)
    if float(src.abs().max()) <= 1e-9 * vmax / min(spacing):
        return None
    info = ops.bicgstab_solve(src, DP, p, spacing, rho, dt, tol, max_it)
    if info.status == L.PF_NONFINITE:
        raise RuntimeError("projection solve: non-finite residual")
    ops.vel_corr(DP, dt / rho, u, v, w, spacing)
    return info


def source_fn(sfsmodel):
    """The face sources of a 'source'-type SFS model as a function of the
    staggered velocity (differentiable when grad mode is on), or None."""
    if sfsmodel is None or getattr(sfsmodel, "modelType", None) != "source":
        return None

    def S(u, v, w):
        sfsmodel.update(u, v, w, requires_grad=torch.is_grad_enabled())
        return sfsmodel.face_sources()
    return S


def rhs_total(state, spacing, mu, rho, sfs=None, source=None):
    """RHS of the velocity: pf_rhs_ns, minus the face sources of a 'source'
    closure evaluated at this state (src/solver/velocity.py:360-383)."""
    k = ops.rhs_ns(*state, spacing, mu, rho, sfs=sfs)
    if source is not None:
        with torch.no_grad():
            fs = source(*state)
        k = tuple(a - b for a, b in zip(k, fs))
    return k


def predictor(state, spacing, mu, rho, dt, sfs=None, source=None, rk4=True):
    """RK4.step / Euler.step composed from RHS evaluations (the reference's
    stage sequence with its stage-4 state u + dt/2 k3), for RHS terms the
    fused predictor kernels do not have."""
    u = tuple(state)
    if not rk4:
        k = rhs_total(u, spacing, mu, rho, sfs, source)
        return tuple(a + b * dt for a, b in zip(u, k))
    h = 0.5 * dt
    ks, cur = [], u
    for s in range(4):
        k = rhs_total(cur, spacing, mu, rho, sfs, source)
        ks.append(k)
        if s < 3:
            cur = tuple((h * kc + uc).contiguous() for kc, uc in zip(k, u))
    return tuple(uc + dt / 6.0 * (((k1 + 2.0 * k2) + 2.0 * k3) + k4)
                 for uc, k1, k2, k3, k4 in zip(u, *ks))


def stage_states(state, spacing, mu, rho, dt, sfs=None, rk4=True, source=None):
    """The predictor's stage states (RK4: u1 = u, u_s = h k_{s-1} + u with
    h = dt/2 for s = 2, 3, 4; Euler: u1 only), recomputed from the step
    input."""
    stages = [tuple(state)]
    if not rk4:
        return stages
    h = 0.5 * dt
    cur = tuple(state)
    for _ in range(3):
        k = rhs_total(cur, spacing, mu, rho, sfs, source)
        cur = tuple((h * kc + uc).contiguous() for kc, uc in zip(k, state))
        stages.append(cur)
    return stages


def _source_vjp(source, stage, kbar):
    """-(dS/du)^T kbar at a stage state; accumulates -(dS/dtheta)^T kbar into
    the closure's parameter gradients (the RHS carries -S)."""
    with torch.enable_grad():
        x = [t.detach().requires_grad_(True) for t in stage]
        fs = source(*x)
        torch.autograd.backward(fs, [-k for k in kbar])
    return tuple(t.grad if t.grad is not None else torch.zeros_like(t) for t in x)


def step_vjp(state, lam_out, spacing, mu, rho, dt, sfs=None, rk4=True,
             tol=1e-12, max_it=20000, source=None):
    """dL/du_n given dL/du_{n+1} (and dL/dF of the SFS stresses if sfs; a
    'source' closure's parameter gradients accumulate in its parameters)."""
    lam = tuple(t.clone() for t in lam_out)
    project(lam, spacing, rho, dt, tol, max_it)            # lam* = P lam
    stages = stage_states(state, spacing, mu, rho, dt, sfs, rk4, source)
    lamF = torch.zeros((6,) + tuple(state[0].shape), dtype=torch.float64,
                       device=state[0].device) if sfs is not None else None
    total = [t.clone() for t in lam]
    if not rk4:
        kbar = tuple(dt * t for t in lam)
        m = rhs_adjoint(stages[0], kbar, spacing, mu, rho)
        if source is not None:
            m = tuple(a + b for a, b in zip(m, _source_vjp(source, stages[0], kbar)))
        if lamF is not None:
            sfs_adjoint_accumulate(kbar, spacing, 1.0, lamF)
        return tuple(a + b for a, b in zip(total, m)), lamF
    h = 0.5 * dt
    wts = (dt / 6.0, dt / 3.0, dt / 3.0, dt / 6.0)
    m_next = None
    for s in (3, 2, 1, 0):
        kbar = tuple(wts[s] * t for t in lam)
        if m_next is not None:
            kbar = tuple(a + h * b for a, b in zip(kbar, m_next))
        m = rhs_adjoint(stages[s], kbar, spacing, mu, rho)
        if source is not None:
            m = tuple(a + b for a, b in zip(m, _source_vjp(source, stages[s], kbar)))
        if lamF is not None:
            sfs_adjoint_accumulate(kbar, spacing, 1.0, lamF)
        total = [a + b for a, b in zip(total, m)]
        m_next = m
    return tuple(total), lamF


class ForwardStep(torch.autograd.Function):
    """One Domain.forwardStep on (u, v, w) as a differentiable map.

    forward: pf_forward_step (FP64, BiCGStab to ``tol``); backward: the
    hand-written adjoint above, recomputing the RK4 stages from the saved
    input.  ``sfs`` (6, nx, ny, nz) stresses, if given, are an input too."""

    @staticmethod
    def forward(ctx, u, v, w, sfs, spacing, mu, rho, dt, rk4, tol, max_it, source=None):
        if sfs is not None:
            sfs = sfs.contiguous()
        ctx.save_for_backward(u, v, w, sfs if sfs is not None else torch.empty(0))
        ctx.cfg = (spacing, mu, rho, dt, rk4, tol, max_it, sfs is not None)
        ctx.source = source
        sd = sfs.detach().contiguous() if sfs is not None else None
        if source is not None:
            # per-stage source closure: composed stages, then the projection
            uo, vo, wo = predictor((u.detach(), v.detach(), w.detach()), spacing, mu, rho,
                                   dt, sd, source, rk4)
            uo, vo, wo = uo.contiguous(), vo.contiguous(), wo.contiguous()
            project((uo, vo, wo), spacing, rho, dt, tol, max_it)
            return uo, vo, wo
        uo, vo, wo = u.detach().clone(), v.detach().clone(), w.detach().clone()
        p = torch.zeros_like(uo)
        DP = torch.zeros_like(uo)
        info = ops.forward_step(uo, vo, wo, p, DP, spacing, mu, rho, dt, rk4=rk4,
                                min_res=tol, max_it=max_it, sfs=sd)
        if info.status == L.PF_NONFINITE:
            raise RuntimeError("forward step: non-finite pressure residual")
        return uo, vo, wo

    @staticmethod
    def backward(ctx, gu, gv, gw):
        u, v, w, sfs = ctx.saved_tensors
        spacing, mu, rho, dt, rk4, tol, max_it, has_sfs = ctx.cfg
        lam = tuple((g if g is not None else torch.zeros_like(u)).contiguous()
                    for g in (gu, gv, gw))
        (lu, lv, lw), lamF = step_vjp((u.detach(), v.detach(), w.detach()), lam,
                                      spacing, mu, rho, dt,
                                      sfs=sfs.detach() if has_sfs else None,
                                      rk4=rk4, tol=tol, max_it=max_it, source=ctx.source)
        return lu, lv, lw, lamF, None, None, None, None, None, None, None, None


def forward_step(u, v, w, spacing, mu, rho, dt, sfs=None, rk4=True, tol=1e-12,
                 max_it=20000, source=None):
    """One differentiable step; ``source`` is a 'source'-closure function
    (source_fn), whose parameter gradients accumulate during backward."""
    return ForwardStep.apply(u, v, w, sfs, tuple(spacing), float(mu), float(rho),
                             float(dt), bool(rk4), float(tol), int(max_it), source)


def _stats_row(it, t, dt, u, v, w, spacing, mu, rho):
    n = u.numel()
    mx = [float(a.abs().max()) for a in (u, v, w)]
    cfl = max(mx[0] / spacing[0], mx[1] / spacing[1], mx[2] / spacing[2]) * dt
    nu = mu / rho
    cfl = max(cfl, max(nu / h ** 2 for h in spacing) * dt)
    tke = float((u * u + v * v + w * w).sum()) / n * 0.5
    div = float(ops.div_vel(u, v, w, spacing).abs().max())
    return (it, t, cfl, mx[0], mx[1], mx[2], tke, div)


def run_training(inputConfig, comms, decomp, geometry, metric, D, startTime):
    """adjointTraining mode of PyFlow.run (src/core/PyFlow.py:312-607).

    numIt steps in windows of numCheckpointIt.  Each window runs forward with
    one checkpoint per step (differentiable steps: pf_forward_step, or the
    composed stages when a 'source' closure is active), then its objective is
    differentiated through the hand-written adjoint:
      * adjointVerification: objective mean(u^2) after the window, with
        ``perturbation`` added to u at the centre cell before the run; returns
        (objective, dL/du at that cell) like the reference (:475-483, 660-663);
      * otherwise: the mean absolute error of u, v, w against the target
        restart file inputConfig.getTargetFileName(startFileIt + itCount)
        (adjoint initial condition sign(u - u_T) / numPoints, :486-533),
        optionally after projecting the target (targetDataVelCorr,
        src/data/domain.py:445-468); the 'source' closure's parameter
        gradients then go to its finalize (gradient averaging, RMSprop,
        learning-rate schedule) and save.
    Constant viscosity; the SFS model, if any, must be 'source'-type or
    none.  Returns None outside verification mode, like the reference."""
    from . import dataReader as dr
    simDt = float(inputConfig.simDt)
    win = int(getattr(inputConfig, "numCheckpointIt", 0) or 0)
    if win <= 0:
        raise Exception("Adjoint training requires specification of numCheckpointIt")
    verification = bool(getattr(inputConfig, "adjointVerification", False))
    sp, mu, rho = tuple(D.spacing), float(D.mu), float(D.rho)
    if D.use_SFSmodel and D.sfsmodel.modelType != "source":
        raise ValueError("adjoint training supports the 'source' ML closure or no SFS model")
    model = D.sfsmodel if D.use_SFSmodel else None
    source = source_fn(model)
    rk4 = D.advancerName == "RK4"
    tol = float(getattr(inputConfig, "min_pressure_residual", 1e-12))
    max_it = int(getattr(inputConfig, "max_pressure_iterations", 20000))
    state = [s.interior() for s in (D.state_u_P, D.state_v_P, D.state_w_P)]
    n = state[0].numel()
    nn = state[0].shape[0] // 2
    if verification:
        state[0][nn, nn, nn] += float(inputConfig.perturbation)
    history, result = [], None
    it, t = 0, float(startTime)
    for _ in range(int(inputConfig.numIt) // win):
        # the velocity carries the graph (the closure's parameters enter
        # through the steps' backward)
        u0 = [x.detach().clone().requires_grad_(True) for x in state]
        cur = tuple(u0)
        for _ in range(win):
            cur = forward_step(*cur, sp, mu, rho, simDt, rk4=rk4, tol=tol, max_it=max_it,
                               source=source)
            it += 1
            t += simDt
            history.append(_stats_row(it, t, simDt, *(c.detach() for c in cur), sp, mu, rho))
        if verification:
            L = torch.mean(cur[0] ** 2)
            L.backward()
            result = (float(L.detach()), float(u0[0].grad[nn, nn, nn]))
        else:
            fname = inputConfig.getTargetFileName(inputConfig.startFileIt + it)
            _, _, tgt = dr.readNGArestart_device(fname, state[0].device, nvar=3)
            if getattr(inputConfig, "targetDataVelCorr", False):
                project(tgt, sp, rho, simDt, tol, max_it, p=D.state_p_P.interior())
            L = sum(torch.sum(torch.abs(c - g)) for c, g in zip(cur, tgt)) / n
            L.backward()
            if model is not None:
                model.finalize(comms)
                if getattr(model, "saveModel", False):
                    model.save()
            history[-1] = history[-1] + (float(L.detach()),)
        for x, c in zip(state, cur):
            x.copy_(c.detach())
    run_training.last_history = history
    return result
