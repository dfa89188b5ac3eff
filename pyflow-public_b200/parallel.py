"""comms / decomp with the reference's interface (src/library/parallel.py).

On one GPU the reference's 2-deep periodic ghost exchange
(``communicate_border``, src/library/parallel.py:301-414) is unnecessary: the
kernels wrap indices.  ``comms`` reduces host scalars across ranks with
torch.distributed when a process group is initialised (gloo or nccl), and is
the identity on one rank, like the reference's single-rank Allreduce.
"""
import numpy as np
import torch
import torch.distributed as dist


class comms:
    """Scalar reductions (src/library/parallel.py:40-112)."""

    def __init__(self, IC=None):
        self.dist = dist.is_available() and dist.is_initialized()
        self.rank = dist.get_rank() if self.dist else 0
        self.size = dist.get_world_size() if self.dist else 1
        self.dtype = getattr(IC, "dtypeNumpy", np.float64)

    def _reduce(self, x, op):
        if self.size == 1:
            return x
        arr = np.atleast_1d(np.asarray(x, dtype=np.float64))
        t = torch.tensor(arr, dtype=torch.float64)
        if dist.get_backend() == "nccl":
            t = t.cuda()
        dist.all_reduce(t, op=op)
        out = t.cpu().numpy()
        return out[0] if np.ndim(x) == 0 else out

    def parallel_sum(self, x):
        return self._reduce(x, dist.ReduceOp.SUM if self.dist else None)

    def parallel_max(self, x):
        return self._reduce(x, dist.ReduceOp.MAX if self.dist else None)

    def parallel_min(self, x):
        return self._reduce(x, dist.ReduceOp.MIN if self.dist else None)

    def finalize(self):
        pass


class decomp:
    """Grid sizes and index ranges (src/library/parallel.py:118-285) for one
    GPU holding the whole periodic box.  The index attributes keep the
    reference's meaning (interior cells imin_..imax_ of an [n+4]^3 array with
    nover = 2) for code that reads them; fields themselves are ghost-free."""

    def __init__(self, IC, config):
        self.prec = getattr(IC, "dtypeTorch", torch.float64)
        self.dtypeNumpy = getattr(IC, "dtypeNumpy", np.float64)
        self.device = torch.device("cuda", torch.cuda.current_device()) \
            if torch.cuda.is_available() else torch.device("cpu")
        self.rank, self.size = 0, 1
        npx = getattr(IC, "nproc_x", 1)
        npy = getattr(IC, "nproc_y", 1)
        npz = getattr(IC, "nproc_z", 1)
        if npx * npy * npz != 1:
            raise ValueError("one GPU holds the whole box: nproc_x*nproc_y*nproc_z "
                             "must be 1 (run replicas for several GPUs)")
        self.npx = self.npy = self.npz = 1
        self.isper = list(getattr(config, "isper", [1, 1, 1]))
        if not all(self.isper):
            raise ValueError("only periodic boxes are supported (the reference's "
                             "working path is periodic)")
        self.nx, self.ny, self.nz = config.Nx, config.Ny, config.Nz
        self.N = self.nx * self.ny * self.nz
        self.nover = 2
        self.nx_, self.ny_, self.nz_ = self.nx, self.ny, self.nz
        self.nxo_, self.nyo_, self.nzo_ = (self.nx + 4, self.ny + 4, self.nz + 4)
        self.imin_loc = self.jmin_loc = self.kmin_loc = 0
        self.imax_loc, self.jmax_loc, self.kmax_loc = self.nx - 1, self.ny - 1, self.nz - 1
        self.imino_ = self.jmino_ = self.kmino_ = 0
        self.imaxo_, self.jmaxo_, self.kmaxo_ = self.nxo_ - 1, self.nyo_ - 1, self.nzo_ - 1
        self.imin_ = self.jmin_ = self.kmin_ = 2
        self.imax_, self.jmax_, self.kmax_ = self.nx + 1, self.ny + 1, self.nz + 1

    def communicate_border(self, A):
        """Periodic ghost refresh of an [n+4]^3 tensor (for callers that still
        hold padded arrays); ghost-free fields need none."""
        if tuple(A.shape) != (self.nxo_, self.nyo_, self.nzo_):
            return
        no = 2
        A[:no] = A[-2 * no:-no]
        A[-no:] = A[no:2 * no]
        A[:, :no] = A[:, -2 * no:-no]
        A[:, -no:] = A[:, no:2 * no]
        A[:, :, :no] = A[:, :, -2 * no:-no]
        A[:, :, -no:] = A[:, :, no:2 * no]

    def free(self):
        pass
