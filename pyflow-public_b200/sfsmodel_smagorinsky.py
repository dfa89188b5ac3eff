"""Smagorinsky eddy viscosity with the reference's interface
(src/sfsmodel/sfsmodel_smagorinsky.py:39-88).

``eddyVisc`` returns mu_t = rho (Cs Delta)^2 |S| at cell centres from the
cell-centred velocity gradients; the fused CUDA kernel (pf_sgs_closure,
model 'smagorinsky') computes gradients, strain magnitude and mu_t in one
pass.  Without an SFS model the reference constructs this class as a blank
placeholder (src/data/domain.py:244-247); so does this package.
"""
from . import ops


class stress_constCs:
    def __init__(self, inputConfig, geo):
        self.modelType = "eddyVisc"
        self.Cs = getattr(inputConfig, "Cs", 0.18)
        fac = getattr(inputConfig, "expFilterFac", 1.0)
        if geo.type != "uniform":
            raise ValueError("sfsmodel_smagorinsky: geometry type not implemented")
        self.Delta = geo.dx * fac
        self.spacing = (geo.dx, geo.dy, geo.dz)

    def eddyVisc(self, state_u, state_v, state_w, rho, metric):
        return ops.sgs_closure("smagorinsky", state_u.interior(), state_v.interior(),
                               state_w.interior(), self.spacing,
                               coef=rho * (self.Cs * self.Delta) ** 2)
