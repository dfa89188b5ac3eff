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


def project(vel, spacing, rho, dt, tol=1e-12, max_it=20000):
    """In-place projection P vel = vel - G L^-1 D vel (FP64 BiCGStab)."""
    u, v, w = vel
    src = ops.div_vel(u, v, w, spacing)
    DP = torch.zeros_like(u)
    p = torch.zeros_like(u)
    info = ops.bicgstab_solve(src, DP, p, spacing, rho, dt, tol, max_it)
    ops.vel_corr(DP, dt / rho, u, v, w, spacing)
    return info


def stage_states(state, spacing, mu, rho, dt, sfs=None, rk4=True):
    """The predictor's stage states (RK4: u1 = u, u_s = h k_{s-1} + u with
    h = dt/2 for s = 2, 3, 4; Euler: u1 only), recomputed from the step
    input."""
    stages = [tuple(state)]
    if not rk4:
        return stages
    h = 0.5 * dt
    cur = tuple(state)
    for _ in range(3):
        k = ops.rhs_ns(*cur, spacing, mu, rho, sfs=sfs)
        cur = tuple(h * kc + uc for kc, uc in zip(k, state))
        stages.append(cur)
    return stages


def step_vjp(state, lam_out, spacing, mu, rho, dt, sfs=None, rk4=True,
             tol=1e-12, max_it=20000):
    """dL/du_n given dL/du_{n+1} (and dL/dF of the SFS stresses if sfs)."""
    lam = tuple(t.clone() for t in lam_out)
    project(lam, spacing, rho, dt, tol, max_it)            # lam* = P lam
    stages = stage_states(state, spacing, mu, rho, dt, sfs, rk4)
    lamF = torch.zeros((6,) + tuple(state[0].shape), dtype=torch.float64,
                       device=state[0].device) if sfs is not None else None
    total = [t.clone() for t in lam]
    if not rk4:
        kbar = tuple(dt * t for t in lam)
        m = rhs_adjoint(stages[0], kbar, spacing, mu, rho)
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
    def forward(ctx, u, v, w, sfs, spacing, mu, rho, dt, rk4, tol, max_it):
        if sfs is not None:
            sfs = sfs.contiguous()
        ctx.save_for_backward(u, v, w, sfs if sfs is not None else torch.empty(0))
        ctx.cfg = (spacing, mu, rho, dt, rk4, tol, max_it, sfs is not None)
        uo, vo, wo = u.detach().clone(), v.detach().clone(), w.detach().clone()
        p = torch.zeros_like(uo)
        DP = torch.zeros_like(uo)
        ops.forward_step(uo, vo, wo, p, DP, spacing, mu, rho, dt, rk4=rk4,
                         min_res=tol, max_it=max_it,
                         sfs=sfs.detach().contiguous() if sfs is not None else None)
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
                                      rk4=rk4, tol=tol, max_it=max_it)
        return lu, lv, lw, lamF, None, None, None, None, None, None, None


def forward_step(u, v, w, spacing, mu, rho, dt, sfs=None, rk4=True, tol=1e-12,
                 max_it=20000):
    return ForwardStep.apply(u, v, w, sfs, tuple(spacing), float(mu), float(rho),
                             float(dt), bool(rk4), float(tol), int(max_it))


def run_training(inputConfig, comms, decomp, geometry, metric, D, startTime):
    """adjointTraining mode of PyFlow.run (src/core/PyFlow.py:312-607):
    numIt steps in windows of numCheckpointIt, each window's objective the
    mean absolute error of the velocity against a target restart file (or
    mean(u^2) in adjointVerification mode), differentiated through the
    hand-written adjoint; returns (objective, gradient at the perturbed cell)
    in verification mode like the reference (src/core/PyFlow.py:660-663)."""
    raise NotImplementedError(
        "adjointTraining through PyFlow.run: use pyflow_b200.adjoint.forward_step "
        "windows (see tests/test_gpu_adjoint.py)")
