"""x-slab decomposition of the periodic box over ranks (one GPU per rank).

Replaces the reference's domain decomposition and ghost exchange (``decomp``
and ``communicate_border``, src/library/parallel.py:118-414) and its scalar
reductions (``comms.parallel_sum`` / ``parallel_max``, :60-94) for boxes
split along x; a step is ``Domain.forwardStep`` (src/data/domain.py:342-402)
in FP64 with the reference's BiCGStab (src/solver/pressure.py:196-297).

Layout: rank r holds planes [x0, x0 + nxl) as a local extended array of
nxl + 2*HALO planes ([nx][ny][nz], z fastest, like every field of the
library): HALO ghost planes, the interior, HALO ghost planes.  Planes are
contiguous, so an exchange sends each neighbour one contiguous block.

A step: exchange u, v, w (HALO = 4 planes: the four RK4 stages each reach one
plane further, so the predictor kernel runs unchanged on the extended array
and is exact on the interior); predictor; exchange u (1 plane); divergence;
the solve (two 1-plane exchanges and three 2-double gathers per iteration,
scalars kept on the device, pf_slab_*); p += DP; exchange DP (1 plane);
projection.  Everything is ordered on the current CUDA stream; the host
reads the solve's stop flag every ``poll`` iterations.

Transports: ``DistSlabs`` (one slab per process over torch.distributed --
NCCL between GPUs, gloo for CPU tensors) and ``LocalSlabs`` (several slabs in
one process on one device, exchanges as device copies), which runs the same
decomposed algorithm where only one GPU is available.
"""
import ctypes

import torch
import torch.distributed as dist

from . import _lib as L
from . import ops

HALO = 4  # ghost planes per side

PF_SLAB_START, PF_SLAB_NEXT, PF_SLAB_APPLY_P, PF_SLAB_S, PF_SLAB_APPLY_S, PF_SLAB_FINAL = range(6)

_lib = L.lib()
_P, _D, _I, _S = ctypes.c_void_p, ctypes.c_double, ctypes.c_int, ctypes.c_size_t
_G = ctypes.POINTER(L.Grid)
for _name, (_args, _res) in {
        "pf_slab_workspace_bytes": ([_G], _S),
        "pf_slab_bicg_vectors": ([_G, _P, ctypes.POINTER(_P), ctypes.POINTER(_P)], _I),
        "pf_slab_bicg_init": ([_G, _I, _D, _D, _D, _I, _P, _P, _P, _S, _P, _P], _I),
        "pf_slab_bicg_phase": ([_G, _I, _I, _P, _I, _P, _P, _P, _P], _I),
        "pf_slab_bicg_info": ([_G, _P, _P, _P], _I),
        "pf_slab_add": ([_G, _I, _P, _P, _P], _I)}.items():
    _fn = getattr(_lib, _name)
    _fn.argtypes = _args
    _fn.restype = _res


def plane_ranges(nx, nranks):
    """(x0, nxl) of every rank: contiguous x planes, the first nx % nranks
    ranks one plane more (the reference's split, src/library/parallel.py:226-235)."""
    if nranks < 1 or nx < nranks:
        raise ValueError("cannot split %d planes over %d ranks" % (nx, nranks))
    base, extra = divmod(nx, nranks)
    out, x0 = [], 0
    for r in range(nranks):
        nxl = base + (1 if r < extra else 0)
        out.append((x0, nxl))
        x0 += nxl
    return out


def extend(field, x0, nxl, halo=HALO):
    """The local extended array of planes [x0 - halo, x0 + nxl + halo) of a
    global periodic field (ghost planes filled with their periodic values)."""
    nx = field.shape[0]
    ix = (torch.arange(nxl + 2 * halo, device=field.device) + (x0 - halo)) % nx
    return field.index_select(0, ix).contiguous()


def _ghost_views(f, nxl, planes, halo):
    """(left interior, right interior, left ghost, right ghost) blocks of
    ``planes`` planes of an extended field."""
    return (f[halo:halo + planes], f[halo + nxl - planes:halo + nxl],
            f[halo - planes:halo], f[halo + nxl:halo + nxl + planes])


class LocalSlabs:
    """Several slabs in one process on one device: rank r's neighbours are
    r - 1 and r + 1 (periodic); an exchange is device copies, a gather is the
    concatenation of the ranks' send buffers in rank order."""

    def __init__(self, nranks):
        self.size = nranks
        self.local_ranks = list(range(nranks))

    def exchange(self, fields, nxls, planes, halo=HALO):
        """fields[r] (list of extended tensors of slab r): fill ``planes``
        ghost planes per side from the neighbours' interior planes."""
        R = self.size
        for r in range(R):
            left, right = (r - 1) % R, (r + 1) % R
            for c, f in enumerate(fields[r]):
                _, _, lg, rg = _ghost_views(f, nxls[r], planes, halo)
                _, lint_right, _, _ = _ghost_views(fields[left][c], nxls[left], planes, halo)
                rint_left, _, _, _ = _ghost_views(fields[right][c], nxls[right], planes, halo)
                lg.copy_(lint_right)
                rg.copy_(rint_left)

    def allgather(self, sends, recvs):
        cat = torch.cat(sends)
        for r in recvs:
            r.copy_(cat)


class DistSlabs:
    """One slab per process over torch.distributed (NCCL for CUDA tensors,
    gloo for CPU ones).  Rank r's left neighbour is r - 1 and its right
    neighbour r + 1 (periodic); an exchange is two send/receive pairs per
    rank, rightward first, each pair matched by order and tag."""

    def __init__(self, group=None):
        self.group = group
        self.size = dist.get_world_size(group)
        self.rank = dist.get_rank(group)
        self.local_ranks = [self.rank]

    def exchange(self, fields, nxls, planes, halo=HALO):
        (mine,), (nxl,) = fields, nxls
        if self.size == 1:
            return LocalSlabs(1).exchange(fields, nxls, planes, halo)
        left = (self.rank - 1) % self.size
        right = (self.rank + 1) % self.size
        gl = (lambda r: dist.get_global_rank(self.group, r)) if self.group is not None else (
            lambda r: r)
        for f in mine:
            lint, rint, lg, rg = _ghost_views(f, nxl, planes, halo)
            ops_ = [dist.P2POp(dist.isend, rint, gl(right), self.group, 0),
                    dist.P2POp(dist.irecv, lg, gl(left), self.group, 0),
                    dist.P2POp(dist.isend, lint, gl(left), self.group, 1),
                    dist.P2POp(dist.irecv, rg, gl(right), self.group, 1)]
            for req in dist.batch_isend_irecv(ops_):
                req.wait()

    def allgather(self, sends, recvs):
        (send,), (recv,) = sends, recvs
        if send.is_cuda:
            dist.all_gather_into_tensor(recv, send, group=self.group)
        else:
            parts = [torch.empty_like(send) for _ in range(self.size)]
            dist.all_gather(parts, send, group=self.group)
            recv.copy_(torch.cat(parts))


class _Slab:
    def __init__(self, x0, nxl, ny, nz, spacing, world, device):
        self.x0, self.nxl = x0, nxl
        shape = (nxl + 2 * HALO, ny, nz)
        self.grid = ops.grid(shape, spacing)
        z = lambda: torch.zeros(shape, dtype=torch.float64, device=device)  # noqa: E731
        self.u, self.v, self.w, self.p, self.DP, self.div = (z() for _ in range(6))
        need = _lib.pf_slab_workspace_bytes(ctypes.byref(self.grid))
        self.ws = torch.empty(need, dtype=torch.uint8, device=device)
        self.send = torch.zeros(2, dtype=torch.float64, device=device)
        self.recv = torch.zeros(2 * world, dtype=torch.float64, device=device)
        self.info = torch.zeros(4, dtype=torch.float64, device=device)
        pp, s = _P(), _P()
        L.check("pf_slab_bicg_vectors", _lib.pf_slab_bicg_vectors(
            ctypes.byref(self.grid), ops._p(self.ws), ctypes.byref(pp), ctypes.byref(s)))
        n = self.grid.nx * ny * nz
        base = self.ws.data_ptr()
        # views of the workspace's exchanged vectors
        self.pp = self.ws.view(torch.float64)[(pp.value - base) // 8:(pp.value - base) // 8 + n] \
            .view(shape)
        self.s = self.ws.view(torch.float64)[(s.value - base) // 8:(s.value - base) // 8 + n] \
            .view(shape)


class SlabDomain:
    """Domain.forwardStep (src/data/domain.py:342-402, RK4, constant
    viscosity, FP64) on an x-slab decomposition.  ``transport`` is a
    DistSlabs (this process holds its rank's slab) or a LocalSlabs (this
    process holds every slab)."""

    def __init__(self, shape, spacing, mu, rho, dt, transport, min_res=1e-10, max_it=20000,
                 poll=4, rk4=True, device="cuda"):
        nx, ny, nz = (int(a) for a in shape)
        self.shape, self.spacing = (nx, ny, nz), tuple(float(h) for h in spacing)
        self.mu, self.rho, self.dt = float(mu), float(rho), float(dt)
        self.min_res, self.max_it, self.poll, self.rk4 = float(min_res), int(max_it), int(poll), rk4
        self.T = transport
        self.ranges = plane_ranges(nx, transport.size)
        if min(n for _, n in self.ranges) < HALO:
            raise ValueError("every slab needs at least %d planes" % HALO)
        self.slabs = [_Slab(*self.ranges[r], ny, nz, spacing, transport.size, device)
                      for r in transport.local_ranks]
        self.nxls = [s.nxl for s in self.slabs]
        self.last_info = None

    # ------------------------------------------------------------ state
    def set_state(self, u, v, w, p=None):
        """Fill the held slabs from global fields (any device)."""
        for s in self.slabs:
            for dst, src in ((s.u, u), (s.v, v), (s.w, w), (s.p, p)):
                if src is None:
                    dst.zero_()
                else:
                    dst.copy_(extend(src.to(dst.device, torch.float64), s.x0, s.nxl))
            s.DP.zero_()

    def interior(self, name):
        """The held slabs' interior planes of field ``name``, in rank order."""
        return [getattr(s, name)[HALO:HALO + s.nxl] for s in self.slabs]

    def gather(self, name):
        """The global field (every slab held here: LocalSlabs)."""
        return torch.cat(self.interior(name))

    # ------------------------------------------------------------ step
    def _xchg(self, names, planes):
        self.T.exchange([[getattr(s, n) for n in names] for s in self.slabs], self.nxls, planes)

    def _gather(self):
        self.T.allgather([s.send for s in self.slabs], [s.recv for s in self.slabs])

    def _phase(self, phase):
        st = torch.cuda.current_stream()
        for s in self.slabs:
            L.check("pf_slab_bicg_phase", _lib.pf_slab_bicg_phase(
                ctypes.byref(s.grid), HALO, phase, ops._p(s.recv), self.T.size, ops._p(s.DP),
                ops._p(s.ws), ops._p(s.send), _P(st.cuda_stream)))

    def solve(self):
        """solver_bicgstab.solve over the slabs: DP from the divergence held
        in ``div``; returns a SolveInfo (max_res, iterations, status)."""
        st = _P(torch.cuda.current_stream().cuda_stream)
        for s in self.slabs:
            L.check("pf_slab_bicg_init", _lib.pf_slab_bicg_init(
                ctypes.byref(s.grid), HALO, self.rho, self.dt, self.min_res, self.max_it,
                ops._p(s.div), ops._p(s.DP), ops._p(s.ws), s.ws.numel(), ops._p(s.send), st))
        self._gather()
        self._phase(PF_SLAB_START)
        it = 0
        while True:
            self._xchg(["pp"], 1)
            self._phase(PF_SLAB_APPLY_P)
            self._gather()
            self._phase(PF_SLAB_S)
            self._xchg(["s"], 1)
            self._phase(PF_SLAB_APPLY_S)
            self._gather()
            self._phase(PF_SLAB_FINAL)
            self._gather()
            self._phase(PF_SLAB_NEXT)
            it += 1
            if it % self.poll == 0 or it >= self.max_it:
                s0 = self.slabs[0]
                L.check("pf_slab_bicg_info", _lib.pf_slab_bicg_info(
                    ctypes.byref(s0.grid), ops._p(s0.ws), ops._p(s0.info), st))
                max_res, iters, status, done = s0.info.tolist()
                if done or it >= self.max_it:
                    break
        info = L.SolveInfo()
        info.max_res, info.iterations, info.outer, info.status = max_res, int(iters), 1, int(status)
        return info

    def forward_step(self):
        """One Domain.forwardStep over the slabs; returns the SolveInfo."""
        sp = self.spacing
        self._xchg(["u", "v", "w"], HALO)
        for s in self.slabs:
            ops.predictor_step(s.u, s.v, s.w, sp, self.mu, self.rho, self.dt, rk4=self.rk4)
        self._xchg(["u"], 1)
        for s in self.slabs:
            ops.div_vel(s.u, s.v, s.w, sp, out=s.div)
        info = self.solve()
        st = _P(torch.cuda.current_stream().cuda_stream)
        for s in self.slabs:
            L.check("pf_slab_add", _lib.pf_slab_add(
                ctypes.byref(s.grid), HALO, ops._p(s.DP), ops._p(s.p), st))
        self._xchg(["DP"], 1)
        for s in self.slabs:
            ops.vel_corr(s.DP, self.dt / self.rho, s.u, s.v, s.w, sp)
        self.last_info = info
        return info
