"""'Gradient' (tensor) SFS model with the reference's interface
(src/sfsmodel/sfsmodel_gradient.py:39-148).

``update`` fills FXX, FYY, FZZ, FXY, FXZ, FYZ = (dx^2/12) du_i/dx_k du_j/dx_k
at cell centres; one fused CUDA kernel (pf_sgs_closure, model 'gradient')
computes the nine cell-centred gradients and the six products.  The
velocity RHS adds these stresses to the viscous flux exactly as the reference
does (src/solver/velocity.py:262-267,286-291,310-315).
"""
from . import ops


class residual_stress:
    def __init__(self, decomp, geo, metric):
        self.modelType = "tensor"
        if geo.type != "uniform":
            raise ValueError("sfsmodel_gradient: geometry type not implemented")
        self.const = geo.dx * geo.dx / 12.0
        self.spacing = (geo.dx, geo.dy, geo.dz)
        self.stacked = None

    def update(self, state_u, state_v, state_w, metric):
        self.stacked = ops.sgs_closure("gradient", state_u.interior(),
                                       state_v.interior(), state_w.interior(),
                                       self.spacing, coef=self.const,
                                       out=self.stacked)
        (self.FXX, self.FYY, self.FZZ, self.FXY, self.FXZ, self.FYZ) = self.stacked.unbind(0)
