"""Pressure Poisson solvers with the reference's interface
(src/solver/pressure.py:44-297).

``solver_bicgstab(...).solve(state_DP_P, state_p_P, source_P)`` solves
(-vol L) DP = -vol rho/dt source from DP = 0 to the reference's max-norm
relative residual, adds DP to p, and returns the residual ratio -- one C-ABI
call (pf_bicgstab_solve).  ``precision='mixed'`` runs the FP32 inner solve
with FP64 refinement instead.  ``solver_jacobi`` keeps the reference's
fixed-sweep Jacobi including its residual ratio and its DP/p convention.
Unlike the reference, ``source_P`` is left unscaled.
"""
from . import _lib as L
from . import ops


class SolverError(RuntimeError):
    """Raised when a solve ends in breakdown or with a non-finite residual
    (the reference exits its loop silently on breakdown,
    src/solver/pressure.py:247-248,266-267; ``raise_on_breakdown=False``
    restores that behaviour)."""


class Pressure_Base:
    def __init__(self, decomp, metric):
        self.decomp = decomp
        self.metric = metric

    def applyOperator(self, A, B):
        """B = (-vol L) A on ghost-free tensors (src/solver/pressure.py:54-84)."""
        ops.laplace_apply(A, self.metric.spacing, out=B)


class solver_bicgstab:
    def __init__(self, comms, decomp, metric, geo, rho, simDt, min_residual,
                 max_iterations, precision="fp64", raise_on_breakdown=False):
        self.comms = comms
        self.pressure = Pressure_Base(decomp, metric)
        self.min_residual = min_residual
        self.max_iterations = max_iterations
        self.rho, self.simDt = rho, simDt
        self.spacing = metric.spacing
        self.vol = metric.vol
        self.precision = precision
        self.raise_on_breakdown = raise_on_breakdown
        self.last_info = None

    def solve(self, state_DP_P, state_p_P, source_P):
        info = ops.bicgstab_solve(source_P, state_DP_P.interior(),
                                  state_p_P.interior(), self.spacing, self.rho,
                                  self.simDt, self.min_residual,
                                  self.max_iterations, prec=self.precision)
        self.last_info = info
        if self.raise_on_breakdown and info.status in (L.PF_BREAKDOWN, L.PF_NONFINITE):
            raise SolverError("BiCGStab: %s after %d iterations"
                              % (L.lib().pf_status_string(info.status).decode(),
                                 info.iterations))
        return info.max_res


class solver_jacobi:
    def __init__(self, comms, decomp, metric, geo, rho, simDt,
                 Num_pressure_iterations):
        self.comms = comms
        self.pressure = Pressure_Base(decomp, metric)
        self.Num_pressure_iterations = Num_pressure_iterations
        self.rho, self.simDt = rho, simDt
        self.spacing = metric.spacing
        if not (abs(geo.dx - geo.dy) <= 1e-12 * geo.dx and abs(geo.dx - geo.dz) <= 1e-12 * geo.dx):
            # the reference's sweep uses h = dx for every direction
            # (src/solver/pressure.py:133,141-147)
            raise ValueError("solver_jacobi assumes dx = dy = dz")

    def solve(self, state_pOld_P, state_p_P, source_P):
        return ops.jacobi_solve(source_P, state_pOld_P.interior(),
                                state_p_P.interior(), self.spacing, self.rho,
                                self.simDt, self.Num_pressure_iterations)
