"""Continuous-batching server for many decaying-turbulence solves.

Requests (grid N^3, seed, viscosity, number of steps) arrive over time.  The
server admits a waiting request as soon as a slot and enough device memory are
free (admission by free HBM: a byte budget, or any callable that reports free
bytes), allocates its fields once and keeps them resident until it is done,
captures its time step as a CUDA graph (pyflow_b200.plan.StepPlan: device-side
convergence loops, no host synchronisation inside a step) and replays that
graph on the request's own stream.  Requests that arrive while others run are
admitted into free slots, and the steps of all active requests are in flight on
the device at the same time.  Each step of a request depends only on its own
buffers, so its result is the same alone and in any mix.

A request's initial field is the seeded k^4 exp(-2 (k/k0)^2) spectrum with
its noise drawn on the device from the request's seed (no host-side random
numbers on the admission path).

Reported: per-request latency (arrival to completion), its p50/p99, and the
aggregate cell-steps/s.
"""
import math
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import initial
from .plan import StepPlan


@dataclass
class Request:
    id: int
    n: int                       # grid is n^3 on [0, 2 pi]^3
    seed: int
    nu: float
    dt: float
    steps: int
    arrival: float = 0.0         # seconds after the server starts
    k0: float = 4.0
    urms: float = 1.0


@dataclass
class Result:
    id: int
    n: int
    steps: int
    arrival: float
    admitted: float
    finished: float
    stats: dict = field(default_factory=dict)
    status: str = "ok"
    error: str = ""
    fields: tuple = None

    @property
    def latency(self):
        return self.finished - self.arrival


def footprint_bytes(n, prec="mixed"):
    """Device bytes one request holds: u, v, w, p, DP (FP64) and its plan
    workspace."""
    import ctypes
    from . import _lib as L
    from . import ops
    from .plan import _lib as PL
    g = ops.grid((n, n, n), (2 * math.pi / n,) * 3)
    ws = PL.pf_step_plan_workspace_bytes(ctypes.byref(g), ops.PREC[prec])
    return 5 * 8 * n ** 3 + ws + 64


class _Slot:
    def __init__(self, req, fields, plan, stream, admitted, nbytes):
        self.req = req
        self.fields = fields
        self.plan = plan
        self.stream = stream
        self.admitted = admitted
        self.launched = 0
        self.event = None
        self.nbytes = nbytes


class Server:
    def __init__(self, max_slots=8, hbm_budget=None, free_hbm=None, prec="mixed",
                 device="cuda", steps_per_launch=1, min_res=1e-10, max_it=20000,
                 keep_fields=False):
        self.device = torch.device(device)
        self.max_slots = max_slots
        self.prec = prec
        self.steps_per_launch = steps_per_launch
        self.min_res, self.max_it = min_res, max_it
        self.keep_fields = keep_fields
        if free_hbm is None:
            if hbm_budget is None:
                free, _ = torch.cuda.mem_get_info(self.device)
                hbm_budget = int(0.8 * free)
            budget = hbm_budget
            self._free = lambda used: budget - used
        else:
            # free_hbm(used_bytes) -> free bytes (e.g. a device query or a fake)
            self._free = free_hbm
        self.max_active = 0
        self._used = 0

    # ------------------------------------------------------------------
    def _admit(self, req, now):
        nbytes = footprint_bytes(req.n, self.prec)
        if nbytes > self._free(self._used):
            return None
        n = req.n
        sp = (2 * math.pi / n,) * 3
        stream = torch.cuda.Stream(self.device)
        with torch.cuda.stream(stream):
            u, v, w = initial.spectral_velocity_device(
                (n, n, n), k0=req.k0, urms=req.urms, seed=req.seed, device=self.device,
                noise="device")
            u, v, w = u.contiguous(), v.contiguous(), w.contiguous()
            p = torch.zeros_like(u)
            DP = torch.zeros_like(u)
        stream.synchronize()
        plan = StepPlan(u, v, w, p, DP, sp, req.nu, 1.0, req.dt, min_res=self.min_res,
                        max_it=self.max_it, prec=self.prec)
        self._used += nbytes
        return _Slot(req, (u, v, w, p, DP), plan, stream, now, nbytes)

    def _release(self, slot):
        slot.plan.close()
        self._used -= slot.nbytes
        slot.fields = None

    def run(self, requests, clock=None):
        """Serve ``requests`` (arrival times in seconds from now); returns the
        results in completion order."""
        clock = clock or time.perf_counter
        pending = sorted(requests, key=lambda r: (r.arrival, r.id))
        active, results = [], []
        t0 = clock()
        while pending or active:
            now = clock() - t0
            # admission: arrived requests into free slots, in arrival order
            while pending and pending[0].arrival <= now and len(active) < self.max_slots:
                req = pending[0]
                if footprint_bytes(req.n, self.prec) > self._free(0):
                    pending.pop(0)   # can never fit: reject, do not block the queue
                    results.append(Result(req.id, req.n, req.steps, req.arrival, now, now,
                                          status="rejected", error="exceeds device memory"))
                    continue
                slot = self._admit(req, now)
                if slot is None:
                    break            # wait for memory to free up
                pending.pop(0)
                active.append(slot)
                self.max_active = max(self.max_active, len(active))
            # advance every active request whose previous launch has finished
            progressed = False
            for slot in list(active):
                if slot.event is not None and not slot.event.query():
                    continue
                if slot.launched < slot.req.steps:
                    k = min(self.steps_per_launch, slot.req.steps - slot.launched)
                    slot.plan.launch(k, stream=slot.stream)
                    slot.launched += k
                    slot.event = torch.cuda.Event()
                    slot.event.record(slot.stream)
                    progressed = True
                    continue
                # all steps done and completed on the device
                st = slot.plan.stats()
                res = Result(slot.req.id, slot.req.n, slot.req.steps, slot.req.arrival,
                             slot.admitted, clock() - t0, stats=st)
                if int(st["status"]) != 0:
                    res.status = "solver-status-%d" % int(st["status"])
                if self.keep_fields:
                    res.fields = tuple(f.clone() for f in slot.fields[:3])
                self._release(slot)
                active.remove(slot)
                results.append(res)
                progressed = True
            if not progressed:
                if active:
                    time.sleep(2e-5)
                elif pending:
                    wait = pending[0].arrival - (clock() - t0)
                    if wait > 0:
                        time.sleep(min(wait, 0.01))
        return results


def assign_requests(requests, free_bytes, prec="mixed"):
    """Shard a request stream over GPUs (one rank each): every request goes,
    in arrival order, to the rank with the least work assigned so far
    (cell-steps), among the ranks whose free HBM can hold it; ties go to the
    rank with more free HBM, then the lower rank.  Requests that fit no rank
    are returned separately.  The assignment is deterministic, so every rank
    computes the same one without communicating.  Returns (per-rank lists,
    unplaceable list)."""
    world = len(free_bytes)
    load = [0] * world
    out = [[] for _ in range(world)]
    rejected = []
    for req in sorted(requests, key=lambda r: (r.arrival, r.id)):
        need = footprint_bytes(req.n, prec)
        cands = [r for r in range(world) if need <= free_bytes[r]]
        if not cands:
            rejected.append(req)
            continue
        r = min(cands, key=lambda k: (load[k], -free_bytes[k], k))
        out[r].append(req)
        load[r] += req.n ** 3 * req.steps
    return out, rejected


def percentile(xs, q):
    xs = sorted(xs)
    if not xs:
        return float("nan")
    k = (len(xs) - 1) * q / 100.0
    f, c = int(math.floor(k)), int(math.ceil(k))
    return xs[f] + (xs[c] - xs[f]) * (k - f)


def stream_requests(count, sizes=(32, 48, 64, 96, 128, 192), steps=50, rate=None,
                    seed0=1000, k0=4.0, rng_seed=7):
    """The decaying-turbulence request stream: N uniform over ``sizes``,
    nu = 0.02 * 32 / N, seeds seed0 + i, Poisson arrivals at ``rate``
    requests/s (all at t = 0 when rate is None).  dt follows a CFL of ~0.3 at
    urms = 1 (the stream's configuration states no dt)."""
    rng = np.random.default_rng(rng_seed)
    t, out = 0.0, []
    for i in range(count):
        n = int(rng.choice(sizes))
        if rate:
            t += rng.exponential(1.0 / rate)
        dx = 2 * math.pi / n
        out.append(Request(id=i, n=n, seed=seed0 + i, nu=0.02 * 32 / n,
                           dt=0.3 * dx / 4.0, steps=steps, arrival=t if rate else 0.0, k0=k0))
    return out


def summarize(results, wall):
    ok = [r for r in results if r.status == "ok"]
    lat = [r.latency for r in ok]
    cells = sum(r.n ** 3 * r.steps for r in ok)
    return {"requests": len(results), "completed": len(ok),
            "p50_latency_s": percentile(lat, 50), "p99_latency_s": percentile(lat, 99),
            "cell_steps_per_s": cells / wall if wall > 0 else float("nan"),
            "wall_s": wall}
