"""Domain with the reference's interface (src/data/domain.py:56-468).

Holds the velocity/pressure states on the device and advances them:
``forwardStep(dt)`` = SFS pre-step (src/data/domain.py:347-355), RK4 or Euler
predictor, and ``velCorr`` (divergence, Poisson solve, projection) once per
step after the predictor (:361-367).  Without an SFS model, or with the
'tensor' models, the whole step is one C-ABI call (pf_forward_step).

Optional configuration keys beyond the reference's:
  precisionMode  'fp64' (default), 'mixed' (FP32 fluxes, stages and inner
                 Poisson solve; FP64 state, residuals, inner products and
                 refinement to the same tolerance) or 'mixed_mg' ('mixed' with
                 the FP32 passes preconditioned by a multigrid V-cycle);
  SFSmodel       also 'MLP' (the 9 -> 128 -> 128 -> 6 BF16 closure in the
                 'tensor' slot, pyflow_b200.sfsmodel_mlp); 'ML' is the
                 reference's 'source' network (pyflow_b200.sfsmodel_ML).
"""
import numpy as np
import torch

from . import advancer, ops, pressure, sfsmodel_gradient, sfsmodel_smagorinsky
from . import state as st
from . import velocity


class Domain:
    def __init__(self, inputConfig, comms, decomp, data_IC, geometry, metric,
                 names, startTime):
        self.inputConfig = inputConfig
        self.decomp = decomp
        self.metric = metric
        self.geometry = geometry
        self.spacing = metric.spacing
        self.equationMode = getattr(inputConfig, "equationMode", "NS")
        if self.equationMode != "NS":
            raise ValueError("equationMode %r not supported (only 'NS')" % self.equationMode)
        self.precision = getattr(inputConfig, "precisionMode", None)
        if self.precision is None:
            self.precision = "mixed" if getattr(inputConfig, "dtypeTorch", torch.float64) == torch.float32 else "fp64"
        simDt = inputConfig.simDt

        self.state_u_P = st.state_P(decomp, data_IC[..., 0])
        self.state_v_P = st.state_P(decomp, data_IC[..., 1])
        self.state_w_P = st.state_P(decomp, data_IC[..., 2])
        self.state_p_P = st.state_P(decomp, data_IC[..., 3])
        self.state_DP_P = st.state_P(decomp, data_IC[..., 3])
        self.state_data_all = (self.state_u_P, self.state_v_P, self.state_w_P,
                               self.state_p_P)
        self.data_all_CPU = st.data_all_CPU(decomp, startTime, simDt, names,
                                            self.state_data_all)
        self.advancerName = inputConfig.advancerName
        if self.advancerName[:-1] == "RK":
            z = np.zeros((decomp.nx_, decomp.ny_, decomp.nz_))
            self.state_uTmp_P = st.state_P(decomp, z)
            self.state_vTmp_P = st.state_P(decomp, z)
            self.state_wTmp_P = st.state_P(decomp, z)
        else:
            self.state_uTmp_P = self.state_vTmp_P = self.state_wTmp_P = None

        self.mu = inputConfig.mu
        self.rho = inputConfig.rho
        self.source_P = torch.zeros(decomp.nx_, decomp.ny_, decomp.nz_,
                                    dtype=torch.float64, device=decomp.device)
        # VISC_P = mu everywhere (src/data/domain.py:130-131); kept as a scalar
        # until an eddy-viscosity model makes it a field
        self.VISC_P = float(self.mu)

        sfs = getattr(inputConfig, "SFSmodel", "none")
        self.use_SFSmodel = True
        if sfs == "Smagorinsky":
            self.sfsmodel = sfsmodel_smagorinsky.stress_constCs(inputConfig, geometry)
        elif sfs == "gradient":
            self.sfsmodel = sfsmodel_gradient.residual_stress(decomp, geometry, metric)
        elif sfs == "MLP":
            from . import sfsmodel_mlp
            self.sfsmodel = sfsmodel_mlp.residual_stress(inputConfig, decomp, geometry)
        elif sfs == "ML":
            from . import sfsmodel_ML
            self.sfsmodel = sfsmodel_ML.residual_stress(inputConfig, decomp, geometry)
        else:
            self.use_SFSmodel = False
            self.sfsmodel = sfsmodel_smagorinsky.stress_constCs(inputConfig, geometry)
        if self.sfsmodel.modelType == "eddyVisc":
            self.muMolec = self.mu

        self.forwardRHS = velocity.ForwardRHS(inputConfig, decomp, metric,
                                              self.rho, self.VISC_P, self.sfsmodel)
        if self.advancerName == "Euler":
            self.forwardAdvancer = advancer.Euler(self.state_u_P, self.state_v_P,
                                                  self.state_w_P, self.forwardRHS)
        elif self.advancerName == "RK4":
            self.forwardAdvancer = advancer.RK4(
                self.state_u_P, self.state_uTmp_P, self.state_v_P, self.state_vTmp_P,
                self.state_w_P, self.state_wTmp_P, self.forwardRHS, prec=self.precision)
        else:
            raise Exception("\n Advancer type " + self.advancerName +
                            " unknown! Options are Euler and RK4.")

        self.doPressure = True
        self.max_resP = 0.0
        self.last_info = None
        mode = getattr(inputConfig, "pSolverMode", "bicgstab")
        self.pSolverMode = mode
        if mode == "Jacobi":
            self.poisson = pressure.solver_jacobi(comms, decomp, metric, geometry,
                                                  inputConfig.rho, simDt,
                                                  inputConfig.max_pressure_iterations)
        elif mode == "bicgstab":
            self.poisson = pressure.solver_bicgstab(
                comms, decomp, metric, geometry, inputConfig.rho, simDt,
                inputConfig.min_pressure_residual,
                inputConfig.max_pressure_iterations, precision=self.precision)
        elif mode == "RedBlackGS":
            raise Exception("\nRed-black GS not yet implemented\n")
        elif mode == "none":
            self.doPressure = False
        else:
            raise ValueError("pSolverMode %r unknown" % mode)

    # ------------------------------------------------------------------
    def _set_visc(self, mu_t):
        if isinstance(self.VISC_P, torch.Tensor):
            self.VISC_P.copy_(self.muMolec + mu_t)
        else:
            self.VISC_P = self.muMolec + mu_t
        for r in (self.forwardRHS.rhs1, getattr(self.forwardRHS, "rhs2", None),
                  getattr(self.forwardRHS, "rhs3", None),
                  getattr(self.forwardRHS, "rhs4", None)):
            if r is not None:
                r.VISC = self.VISC_P

    def forwardStep(self, simDt):
        """src/data/domain.py:342-367"""
        if self.use_SFSmodel:
            if self.sfsmodel.modelType == "eddyVisc":
                muEddy = self.sfsmodel.eddyVisc(self.state_u_P, self.state_v_P,
                                                self.state_w_P, self.rho, self.metric)
                self._set_visc(muEddy)
            elif self.sfsmodel.modelType == "tensor":
                self.sfsmodel.update(self.state_u_P, self.state_v_P,
                                     self.state_w_P, self.metric)
        fused = (self.doPressure and isinstance(self.forwardRHS, velocity.ForwardRHS)
                 and self.sfsmodel.modelType != "source")
        if fused:
            mu, visc = velocity.visc_args(self.VISC_P)
            sfs = velocity.sfs_args(self.sfsmodel) if self.use_SFSmodel else None
            if self.precision != "fp64":
                # the mixed forms' stages read the closure fields in FP32
                visc = None if visc is None else visc.float()
                sfs = None if sfs is None else sfs.float()
            solver = "bicgstab" if self.pSolverMode == "bicgstab" else "jacobi"
            p = self.poisson
            max_it = (p.max_iterations if solver == "bicgstab"
                      else p.Num_pressure_iterations)
            min_res = p.min_residual if solver == "bicgstab" else 0.0
            info = ops.forward_step(
                self.state_u_P.interior(), self.state_v_P.interior(),
                self.state_w_P.interior(), self.state_p_P.interior(),
                self.state_DP_P.interior(), self.spacing, mu, self.rho, simDt,
                rk4=(self.advancerName == "RK4"), solver=solver, min_res=min_res,
                max_it=max_it, prec=self.precision, visc=visc, sfs=sfs)
            self.last_info = info
            self.max_resP = info.max_res
            return
        self.forwardAdvancer.step(simDt)
        if self.doPressure:
            self.velCorr(simDt)

    def velCorr(self, simDt):
        """src/data/domain.py:373-402"""
        self.metric.div_vel(self.state_u_P, self.state_v_P, self.state_w_P,
                            self.source_P)
        self.max_resP = self.poisson.solve(self.state_DP_P, self.state_p_P,
                                           self.source_P)
        self.last_info = getattr(self.poisson, "last_info", None)
        ops.vel_corr(self.state_DP_P.interior(), simDt / self.rho,
                     self.state_u_P.interior(), self.state_v_P.interior(),
                     self.state_w_P.interior(), self.spacing)
