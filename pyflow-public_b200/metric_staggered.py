"""metric_uniform with the reference's interface
(src/metric/metric_staggered.py:38-800).

The staggered operators that sit on the hot path run as CUDA kernels through
the C ABI: the divergence (div_vel) and the 7-point Laplacian.  The remaining
methods that the SGS closures and the projection use (cell-centred velocity
gradients, the pressure gradient) keep the reference's formulas as short
torch expressions on ghost-free tensors with periodic rolls.
"""
import torch

from . import ops


def _fwd(f, dim):
    # f[i+1] - f[i] along dim (periodic)
    return torch.roll(f, -1, dim) - f


def _bwd(f, dim):
    # f[i] - f[i-1] along dim (periodic)
    return f - torch.roll(f, 1, dim)


class metric_uniform:
    def __init__(self, geo):
        if geo.type != "uniform":
            raise ValueError("grid type not implemented")
        self.geo = geo
        self.spacing = (geo.dx, geo.dy, geo.dz)
        self.grad_x = self.div_x = geo.dxi
        self.grad_y = self.div_y = geo.dyi
        self.grad_z = self.div_z = geo.dzi
        self.interp_x = self.interp_y = self.interp_z = 0.5
        self.vol = geo.dx * geo.dy * geo.dz
        for a in ("imin_", "imax_", "jmin_", "jmax_", "kmin_", "kmax_"):
            setattr(self, a, getattr(geo, a))

    @property
    def Laplace(self):
        """The reference's per-cell coefficient array (metric_staggered.py:84-102)
        reduced to its 3x3 uniform values: rows x, y, z; columns -1, 0, +1."""
        c = []
        for di in (self.geo.dxi, self.geo.dyi, self.geo.dzi):
            c.append([(di * di) * (-1.0 * self.vol), ((-2.0 * di) * di) * (-1.0 * self.vol),
                      (di * di) * (-1.0 * self.vol)])
        return torch.tensor(c, dtype=torch.float64)

    # ---- hot-path operators (CUDA) ------------------------------------
    def div_vel(self, state_u, state_v, state_w, divg):
        """Divergence at cell centres (metric_staggered.py:438-453)."""
        ops.div_vel(state_u.interior(), state_v.interior(), state_w.interior(),
                    self.spacing, out=divg)

    def apply_laplace(self, A, out=None):
        """(-vol L) A, Pressure_Base.applyOperator (src/solver/pressure.py:54-84)."""
        return ops.laplace_apply(A, self.spacing, out=out)

    # ---- other operators ------------------------------------------------
    def grad_P(self, state):
        """Backward differences to faces (metric_staggered.py:390-401)."""
        p = state.interior()
        state.grad_x = _bwd(p, 0) * self.grad_x
        state.grad_y = _bwd(p, 1) * self.grad_y
        state.grad_z = _bwd(p, 2) * self.grad_z

    def grad_vel_center(self, state, comp):
        """Cell-centred velocity gradients (metric_staggered.py:215-268):
        the normal derivative is a one-sided difference of the face values,
        the transverse ones are central differences of the face-to-centre
        interpolant, evaluated with periodic wrap everywhere."""
        f = state.interior()
        d = {"u": 0, "v": 1, "w": 2}[comp]
        hs = (self.grad_x, self.grad_y, self.grad_z)
        c = 0.5 * (torch.roll(f, -1, d) + f)  # value at the cell centre
        g = [None, None, None]
        for e in range(3):
            if e == d:
                g[e] = _fwd(f, e) * hs[e]
            else:
                fc = 0.5 * (c + torch.roll(c, 1, e))       # interp to faces
                g[e] = (torch.roll(fc, -1, e) - fc) * hs[e]
        state.grad_x, state.grad_y, state.grad_z = g
