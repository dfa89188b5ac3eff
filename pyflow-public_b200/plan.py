"""Graph-captured time steps (pf_step_plan_*).

A StepPlan binds one set of device fields (u, v, w, p, DP) and captures a whole
Domain.forwardStep -- predictor, divergence, Poisson solve with device-side
convergence loops, projection and the monitor statistics -- as one CUDA graph.
``launch(n)`` enqueues n steps without any host synchronisation; ``stats()``
reads the last step's statistics (max|u|, max|v|, max|w|, TKE, max|div u|,
max_res, iterations, status).
"""
import ctypes

import torch

from . import _lib as L
from . import ops

_lib = L.lib()
_lib.pf_step_plan_workspace_bytes.argtypes = [ctypes.POINTER(L.Grid), ctypes.c_int]
_lib.pf_step_plan_workspace_bytes.restype = ctypes.c_size_t
_lib.pf_step_plan_create.argtypes = [
    ctypes.POINTER(L.Grid), ctypes.c_int, ctypes.c_int] + [ctypes.c_void_p] * 5 + [
    ctypes.c_double] * 4 + [ctypes.c_int, ctypes.c_void_p, ctypes.c_size_t,
                            ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]
_lib.pf_step_plan_create.restype = ctypes.c_int


class StepClosure(ctypes.Structure):
    """pf_step_closure (include/pyflow_b200.h)."""
    _fields_ = [("kind", ctypes.c_int), ("coef", ctypes.c_double), ("wpack", ctypes.c_void_p),
                ("err", ctypes.c_void_p), ("field", ctypes.c_void_p),
                ("field_bytes", ctypes.c_size_t)]


for _fn in (_lib.pf_step_closure_bytes, _lib.pf_step_closure_stage_offset):
    _fn.argtypes = [ctypes.POINTER(L.Grid), ctypes.c_int, ctypes.c_int]
    _fn.restype = ctypes.c_size_t
_lib.pf_step_plan_create_sfs.argtypes = [
    ctypes.POINTER(L.Grid), ctypes.c_int, ctypes.c_int] + [ctypes.c_void_p] * 5 + [
    ctypes.c_double] * 4 + [ctypes.c_int, ctypes.POINTER(StepClosure), ctypes.c_void_p,
                            ctypes.c_size_t, ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]
_lib.pf_step_plan_create_sfs.restype = ctypes.c_int
_lib.pf_step_plan_launch.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
_lib.pf_step_plan_launch.restype = ctypes.c_int
_lib.pf_step_plan_destroy.argtypes = [ctypes.c_void_p]
_lib.pf_step_plan_destroy.restype = ctypes.c_int

class BatchMember(ctypes.Structure):
    _fields_ = [("grid", L.Grid)] + [(n, ctypes.c_void_p) for n in ("u", "v", "w", "p", "DP")] + [
        ("mu", ctypes.c_double), ("rho", ctypes.c_double), ("dt", ctypes.c_double),
        ("min_res", ctypes.c_double), ("max_it", ctypes.c_int), ("fresh", ctypes.c_int),
        ("ws", ctypes.c_void_p),
        ("ws_bytes", ctypes.c_size_t), ("stats", ctypes.c_void_p)]


_lib.pf_batch_table_bytes.argtypes = [ctypes.c_int]
_lib.pf_batch_table_bytes.restype = ctypes.c_size_t
_lib.pf_batch_plan_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(BatchMember),
                                      ctypes.c_int, ctypes.c_void_p, ctypes.c_size_t,
                                      ctypes.POINTER(ctypes.c_void_p)]
_lib.pf_batch_plan_create.restype = ctypes.c_int
MAX_BATCH = 64

# SFS closures a plan can evaluate inside its graph (pf_step_plan_create_sfs)
CLOSURES = {"smagorinsky": 1, "gradient": 2, "mlp": 3}

STAT_NAMES = ("max_u", "max_v", "max_w", "tke", "max_div", "max_res",
              "iterations", "status", "total_iterations", "steps")


class StepPlan:
    """One field set's step graph.  ``closure`` adds the SFS pre-step of
    Domain.forwardStep (src/data/domain.py:347-355) to the graph:
    'smagorinsky' or 'gradient' with its ``coef`` as for ops.sgs_closure, or
    'mlp' with coef = Delta^2, the packed network ``wpack`` and an int32
    error flag ``err`` (sfsmodel_mlp.closure).  The field the stages read
    (the viscosity mu + coef|S|, or the six stresses) is ``self.cfield``, in
    the stages' type."""

    def __init__(self, u, v, w, p, DP, spacing, mu, rho, dt, min_res=1e-10,
                 max_it=20000, prec="fp64", rk4=True, closure=None, coef=0.0, wpack=None,
                 err=None):
        for t, nm in ((u, "u"), (v, "v"), (w, "w"), (p, "p"), (DP, "DP")):
            ops._check(t, u.shape, torch.float64, nm)
        self.fields = (u, v, w, p, DP)
        self.grid = ops.grid(u.shape, spacing)
        pr = ops.PREC[prec]
        need = _lib.pf_step_plan_workspace_bytes(ctypes.byref(self.grid), pr)
        self.ws = torch.empty(need, dtype=torch.uint8, device=u.device)
        self.stats_dev = torch.zeros(10, dtype=torch.float64, device=u.device)
        self.cells = u.numel()
        self._h = ctypes.c_void_p(0)
        self.cfield = None
        if closure is not None:
            kind = CLOSURES[closure]
            g = ctypes.byref(self.grid)
            nbytes = _lib.pf_step_closure_bytes(g, pr, kind)
            off = _lib.pf_step_closure_stage_offset(g, pr, kind)
            self.cbuf = torch.empty(nbytes, dtype=torch.uint8, device=u.device)
            sdt = torch.float64 if pr == L.PF_FP64 else torch.float32
            shape = tuple(u.shape) if kind == 1 else (6,) + tuple(u.shape)
            count = 1
            for a in shape:
                count *= a
            self.cfield = self.cbuf[off:].view(sdt)[:count].view(shape)
            if kind == 3:
                self.err = err if err is not None else torch.zeros(1, dtype=torch.int32,
                                                                   device=u.device)
                self.wpack = wpack
            self.closure = StepClosure(kind, float(coef),
                                       ops._p(wpack) if kind == 3 else None,
                                       ops._p(self.err) if kind == 3 else None,
                                       ops._p(self.cbuf), nbytes)
        # the fields must be ready: wait for the stream that produced them
        torch.cuda.current_stream(u.device).synchronize()
        common = (ctypes.byref(self.grid), pr, 1 if rk4 else 0,
                  *(ops._p(t) for t in self.fields), float(mu), float(rho), float(dt),
                  float(min_res), int(max_it))
        tail = (ops._p(self.ws), self.ws.numel(), ops._p(self.stats_dev), ctypes.byref(self._h))
        if closure is None:
            L.check("pf_step_plan_create", _lib.pf_step_plan_create(*common, *tail))
        else:
            L.check("pf_step_plan_create_sfs", _lib.pf_step_plan_create_sfs(
                *common, ctypes.byref(self.closure), *tail))

    def launch(self, nsteps=1, stream=None):
        s = stream if stream is not None else torch.cuda.current_stream(self.ws.device)
        L.check("pf_step_plan_launch", _lib.pf_step_plan_launch(
            self._h, int(nsteps), ctypes.c_void_p(s.cuda_stream)))

    def reset_counters(self):
        self.stats_dev[8:].zero_()

    def stats(self):
        return dict(zip(STAT_NAMES, self.stats_dev.cpu().tolist()))

    def close(self):
        if self._h and self._h.value:
            _lib.pf_step_plan_destroy(self._h)
            self._h = ctypes.c_void_p(0)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Member:
    """One request of a BatchPlan: its device fields u, v, w, p, DP (FP64,
    one grid), constants, plan workspace and statistics buffer (the layout of
    StepPlan.stats_dev).  The buffers stay owned by the member, so a member
    can move from one batch to the next with its state and running totals."""

    def __init__(self, u, v, w, p, DP, spacing, mu, rho, dt, min_res=1e-10, max_it=20000,
                 prec="mixed_mg"):
        for t, nm in ((u, "u"), (v, "v"), (w, "w"), (p, "p"), (DP, "DP")):
            ops._check(t, u.shape, torch.float64, nm)
        self.fields = (u, v, w, p, DP)
        self.grid = ops.grid(u.shape, spacing)
        self.prec = prec
        need = _lib.pf_step_plan_workspace_bytes(ctypes.byref(self.grid), ops.PREC[prec])
        self.ws = torch.empty(need, dtype=torch.uint8, device=u.device)
        self.stats_dev = torch.zeros(10, dtype=torch.float64, device=u.device)
        self.consts = (float(mu), float(rho), float(dt), float(min_res), int(max_it))
        self.cells = u.numel()
        self.fresh = True
        # the fields must be ready before a plan first uses them
        torch.cuda.current_stream(u.device).synchronize()

    def stats(self):
        return dict(zip(STAT_NAMES, self.stats_dev.cpu().tolist()))

    def c_struct(self):
        mu, rho, dt, min_res, max_it = self.consts
        return BatchMember(self.grid, *(ops._p(t) for t in self.fields), mu, rho, dt, min_res,
                           max_it, 1 if self.fresh else 0, ops._p(self.ws), self.ws.numel(),
                           ops._p(self.stats_dev))


class BatchPlan:
    """One CUDA graph that advances every member by one time step per
    replay (pf_batch_plan_create): the RK4 stages of all members as one
    grouped launch per stage, then each member's divergence, pressure solve,
    projection and statistics as independent graph branches.  Members keep
    their results exactly as with their own StepPlan."""

    def __init__(self, members, rk4=True):
        if not members or len(members) > MAX_BATCH:
            raise ValueError("a batch holds 1..%d members" % MAX_BATCH)
        prec = members[0].prec
        if any(m.prec != prec for m in members):
            raise ValueError("all members of a batch use one precision form")
        self.device = members[0].ws.device
        self.members = list(members)
        # per-member arguments of the grouped launches (first int: error flag)
        self.table = torch.empty(_lib.pf_batch_table_bytes(len(members)), dtype=torch.uint8,
                                 device=self.device)
        arr = (BatchMember * len(members))(*(m.c_struct() for m in members))
        self._h = ctypes.c_void_p(0)
        L.check("pf_batch_plan_create", _lib.pf_batch_plan_create(
            ops.PREC[prec], 1 if rk4 else 0, arr, len(members), ops._p(self.table),
            self.table.numel(), ctypes.byref(self._h)))
        for m in members:
            m.fresh = False

    def launch(self, nsteps=1, stream=None):
        s = stream if stream is not None else torch.cuda.current_stream(self.device)
        L.check("pf_step_plan_launch", _lib.pf_step_plan_launch(
            self._h, int(nsteps), ctypes.c_void_p(s.cuda_stream)))

    def error(self):
        """True if a grouped launch found a tile outside every member's range."""
        return bool(self.table[:4].view(torch.int32).item())

    def close(self):
        if self._h and self._h.value:
            _lib.pf_step_plan_destroy(self._h)
            self._h = ctypes.c_void_p(0)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class StepPipeline:
    """Independent time steps on states that arrive in pinned host memory
    (a request stream), with the host<->device copies overlapped with the
    computation: ``nsets`` field sets with one captured StepPlan each are
    used in turn; host->device copies run on one copy stream and
    device->host copies on another (the two copy engines), so the input of
    request k+1 and the output of request k-1 move while request k computes.
    A set is reused only after its previous request has been copied out, so
    with two sets every pair of requests waits for one chain copy-in ->
    step -> copy-out; three sets (the default) break that chain when the
    copies take longer than the step, and the copy directions bound the rate.
    Ordering is by events only; nothing here synchronises the host.

    ``submit(u, v, w, p, stats_out, state_out=None)`` takes pinned host FP64
    tensors of the grid's shape and a pinned host FP64 tensor of 10 for the
    step's statistics (the layout of ``StepPlan.stats_dev``); with
    ``state_out`` (four pinned host tensors) the advanced u, v, w, p are
    copied back too.  The host tensors must stay untouched until
    ``synchronize()`` (or a later event) shows the request done.  DP starts
    from zero for every request, as in Domain.forwardStep.  ``start(event)``
    makes the copy streams wait for an event of the caller (e.g. the start of
    a timed region) and ``finish(stream)`` makes ``stream`` wait for all
    submitted work.
    """

    def __init__(self, shape, spacing, mu, rho, dt, min_res=1e-10, max_it=20000,
                 prec="fp64", rk4=True, device="cuda", stream=None, nsets=3):
        dev = torch.device(device)
        if nsets < 1:
            raise ValueError("nsets must be at least 1")
        self.nsets = nsets
        self.sets = [[torch.zeros(shape, dtype=torch.float64, device=dev) for _ in range(5)]
                     for _ in range(nsets)]
        self.plans = [StepPlan(*f, spacing, mu, rho, dt, min_res=min_res, max_it=max_it,
                               prec=prec, rk4=rk4) for f in self.sets]
        self.compute = stream if stream is not None else torch.cuda.current_stream(dev)
        self.h2d = torch.cuda.Stream(dev)
        self.d2h = torch.cuda.Stream(dev)
        self.ready = [torch.cuda.Event() for _ in range(nsets)]
        self.done = [torch.cuda.Event() for _ in range(nsets)]
        self.free = [torch.cuda.Event() for _ in range(nsets)]
        for e in self.free:
            e.record(self.compute)
        self.k = 0

    def start(self, event):
        self.h2d.wait_event(event)
        self.d2h.wait_event(event)

    def submit(self, u, v, w, p, stats_out, state_out=None):
        s = self.k % self.nsets
        f = self.sets[s]
        # the set is free once its previous request has computed and copied out
        self.h2d.wait_event(self.free[s])
        with torch.cuda.stream(self.h2d):
            for d, h in zip(f[:4], (u, v, w, p)):
                d.copy_(h, non_blocking=True)
        self.ready[s].record(self.h2d)
        self.compute.wait_event(self.ready[s])
        with torch.cuda.stream(self.compute):
            f[4].zero_()
        self.plans[s].launch(1, stream=self.compute)
        self.done[s].record(self.compute)
        self.d2h.wait_event(self.done[s])
        with torch.cuda.stream(self.d2h):
            stats_out.copy_(self.plans[s].stats_dev, non_blocking=True)
            if state_out is not None:
                for h, d in zip(state_out, f[:4]):
                    h.copy_(d, non_blocking=True)
        self.free[s].record(self.d2h)
        self.k += 1

    def finish(self, stream):
        stream.wait_stream(self.h2d)
        stream.wait_stream(self.d2h)
        stream.wait_stream(self.compute)

    def synchronize(self):
        self.compute.synchronize()
        self.h2d.synchronize()
        self.d2h.synchronize()

    def close(self):
        for pl in self.plans:
            pl.close()
