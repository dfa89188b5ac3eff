"""state_P with the reference's interface (src/data/state.py:98-211).

A state is one ghost-free FP64 device tensor ``interior()`` of shape
(nx, ny, nz); the reference's [n+4]^3 ``var`` with periodic ghosts is
available read-only as ``var`` (a padded copy), and ``update_border`` is a
no-op because the kernels wrap indices.
"""
import numpy as np
import torch


class state_P:
    def __init__(self, decomp, IC=None, need_gradients=True):
        self.decomp = decomp
        self.nover = decomp.nover
        for a in ("imin_", "imax_", "jmin_", "jmax_", "kmin_", "kmax_", "imino_",
                  "imaxo_", "jmino_", "jmaxo_", "kmino_", "kmaxo_"):
            setattr(self, a, getattr(decomp, a))
        self.data = torch.zeros(decomp.nx_, decomp.ny_, decomp.nz_,
                                dtype=torch.float64, device=decomp.device)
        if isinstance(IC, torch.Tensor):
            self.data.copy_(IC)
        elif IC is not None and np.any(IC):
            self.data.copy_(torch.as_tensor(np.asarray(IC, dtype=np.float64)))
        self.grad_x = self.grad_y = self.grad_z = None

    def interior(self):
        return self.data

    @property
    def var(self):
        """Padded [n+4]^3 copy with periodic ghost layers (read-only)."""
        d = self.data
        return torch.nn.functional.pad(d[None, None], (2, 2, 2, 2, 2, 2),
                                       mode="circular")[0, 0]

    def update_border(self):
        pass

    def update_border_i(self):
        pass

    def ZAXPY(self, A, X, Y):
        # Z = A*X + Y (src/data/state.py:157-165)
        self.data.copy_(A * X + Y)

    def copy(self, input):
        self.data.copy_(input)

    def update(self, input):
        self.copy(input)

    def vel_corr(self, inGrad, inScalar):
        # var -= inScalar * inGrad (src/data/state.py:198-211)
        self.data.sub_(inGrad, alpha=inScalar)


class data_all_CPU:
    """Host mirror used for restart I/O (src/data/state.py:38-94)."""

    def __init__(self, decomp, time, dt, names, state_data_all):
        self.nx, self.ny, self.nz = decomp.nx, decomp.ny, decomp.nz
        self.time, self.dt = time, dt
        self.names = list(names)
        self.nvar = len(names)
        self.states = list(state_data_all)
        self.nvar_read = len(self.states)

    def append(self, ivar, inData):
        if ivar < self.nvar_read:
            self.states[ivar].data.copy_(torch.as_tensor(np.asarray(inData, dtype=np.float64)))

    def read(self, ivar):
        if ivar < self.nvar_read:
            return self.states[ivar].data.cpu().numpy()

    def absmax(self, ivar):
        if ivar < self.nvar_read:
            return float(self.states[ivar].data.abs().max())
