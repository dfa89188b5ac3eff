"""Forward right-hand side with the reference's interface
(src/solver/velocity.py:45-383).

``rhs_NavierStokes.evaluate(u, v, w)`` fills ``rhs_u/rhs_v/rhs_w`` through the
C ABI (pf_rhs_ns): viscous + convective staggered fluxes in the reference's
operation order, plus the 'tensor' SFS stresses when the model provides them.
"""
import torch

from . import ops


class ForwardRHS:
    """src/solver/velocity.py:45-76 (Navier-Stokes mode only; the reference's
    scalar mode is broken: it uses undefined names at :54-58)."""

    def __init__(self, inputConfig, decomp, metric, rho, VISC, sfsmodel):
        mode = getattr(inputConfig, "equationMode", "NS")
        if mode != "NS":
            raise ValueError("equationMode %r not supported (only 'NS')" % mode)
        self.rhs1 = rhs_NavierStokes(decomp, metric, rho, VISC, sfsmodel)
        if inputConfig.advancerName[:-1] == "RK":
            self.rhs2 = rhs_NavierStokes(decomp, metric, rho, VISC, sfsmodel)
            self.rhs3 = rhs_NavierStokes(decomp, metric, rho, VISC, sfsmodel)
            self.rhs4 = rhs_NavierStokes(decomp, metric, rho, VISC, sfsmodel)


def visc_args(VISC, mu_default=None):
    """(mu, visc tensor or None): a float VISC or a constant field is passed as
    the scalar mu so the kernels read no viscosity field."""
    if isinstance(VISC, torch.Tensor):
        if getattr(VISC, "_pf_constant", None) is not None:
            return VISC._pf_constant, None
        return 0.0, VISC
    return float(VISC if mu_default is None else mu_default), None


def sfs_args(sfsmodel):
    """Stacked 'tensor' SFS stresses [FXX,FYY,FZZ,FXY,FXZ,FYZ] or None."""
    if sfsmodel is None or getattr(sfsmodel, "modelType", None) != "tensor":
        return None
    st = getattr(sfsmodel, "stacked", None)
    if st is not None:
        return st
    return torch.stack([sfsmodel.FXX, sfsmodel.FYY, sfsmodel.FZZ,
                        sfsmodel.FXY, sfsmodel.FXZ, sfsmodel.FYZ]).contiguous()


class rhs_NavierStokes:
    def __init__(self, decomp, metric, rho, VISC, sfsmodel):
        shape = (decomp.nx_, decomp.ny_, decomp.nz_)
        self.rhs_u = torch.zeros(shape, dtype=torch.float64, device=decomp.device)
        self.rhs_v = torch.zeros_like(self.rhs_u)
        self.rhs_w = torch.zeros_like(self.rhs_u)
        self.metric = metric
        self.rho = rho
        self.VISC = VISC
        self.sfsmodel = sfsmodel

    def evaluate(self, state_u, state_v, state_w):
        mu, visc = visc_args(self.VISC)
        ops.rhs_ns(state_u.interior(), state_v.interior(), state_w.interior(),
                   self.metric.spacing, mu, self.rho, visc=visc,
                   sfs=sfs_args(self.sfsmodel),
                   out=(self.rhs_u, self.rhs_v, self.rhs_w))
        if getattr(self.sfsmodel, "modelType", None) == "source":
            # 'source' closures are evaluated at every stage's state and
            # subtracted on the faces (src/solver/velocity.py:360-383)
            self.sfsmodel.update(state_u.interior(), state_v.interior(), state_w.interior())
            fu, fv, fw = self.sfsmodel.face_sources()
            self.rhs_u.sub_(fu)
            self.rhs_v.sub_(fv)
            self.rhs_w.sub_(fw)
