"""Continuous-batching server for many decaying-turbulence solves.

Requests (grid N^3, seed, viscosity, number of steps) arrive over time.  The
server admits a waiting request as soon as a slot is free and the device has
room for it -- free HBM is queried live at every admission (the device's free
memory plus what torch's caching allocator holds unused), or given by a byte
budget or any callable -- allocates its fields once and keeps them resident
until it is done.

Batched mode (default): all active requests advance together.  One captured
CUDA graph (plan.BatchPlan, pf_batch_plan_create) advances every active
request by one time step per replay: the RK4 stages of all of them run as one
grouped, persistent launch per stage, then each request's divergence,
pressure solve (device-side convergence loops), projection and statistics run
as independent branches of the graph, so their work overlaps on the device.
When a request finishes or a new one is admitted the batch graph is rebuilt
for the new active set (members carry their state over); up to two replays are
in flight, so the host prepares the next one while the device computes.
Per-request mode (batched=False): one StepPlan graph per request, replayed on
the request's own stream.

Each step of a request depends only on its own buffers and runs exactly the
kernels of its own StepPlan, so its result is the same alone and in any mix.

A request's initial field is the seeded k^4 exp(-2 (k/k0)^2) spectrum with
its noise drawn on the device from the request's seed (no host-side random
numbers on the admission path).

Reported: per-request latency (arrival to completion), its p50/p99, and the
aggregate cell-steps/s.
"""
import collections
import math
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import initial
from .plan import BatchPlan, Member, StepPlan


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


def footprint_bytes(n, prec="mixed_mg"):
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


def device_free_bytes(device):
    """Free device memory this process can still use: the device's free
    memory plus the blocks torch's caching allocator holds unused."""
    free, _ = torch.cuda.mem_get_info(device)
    return free + torch.cuda.memory_reserved(device) - torch.cuda.memory_allocated(device)


class Server:
    def __init__(self, max_slots=8, hbm_budget=None, free_hbm=None, prec="mixed_mg",
                 device="cuda", steps_per_launch=1, min_res=1e-10, max_it=20000,
                 keep_fields=False, batched=True, reserve=0.1):
        self.device = torch.device(device)
        self.max_slots = max_slots
        self.prec = prec
        self.steps_per_launch = steps_per_launch
        self.min_res, self.max_it = min_res, max_it
        self.keep_fields = keep_fields
        self.batched = batched
        # _free(used): bytes free for a new request now; _capacity(): bytes a
        # request could ever get (all active requests gone)
        if free_hbm is not None:
            # free_hbm(used_bytes) -> free bytes (e.g. a fake for tests)
            self._free = free_hbm
            self._capacity = lambda: free_hbm(0)
        elif hbm_budget is not None:
            budget = hbm_budget
            self._free = lambda used: budget - used
            self._capacity = lambda: budget
        else:
            # live query at every admission, keeping a reserve of the
            # device's memory for the graphs and the allocator's slack
            total = torch.cuda.get_device_properties(self.device).total_memory
            keep = int(reserve * total)
            self._free = lambda used: device_free_bytes(self.device) - keep
            self._capacity = lambda: device_free_bytes(self.device) - keep + self._used
        self.max_active = 0
        self.rebuilds = 0
        self._used = 0

    # ------------------------------------------------------------------
    def _fields(self, req, stream):
        n = req.n
        with torch.cuda.stream(stream):
            u, v, w = initial.spectral_velocity_device(
                (n, n, n), k0=req.k0, urms=req.urms, seed=req.seed, device=self.device,
                noise="device")
            u, v, w = u.contiguous(), v.contiguous(), w.contiguous()
            p = torch.zeros_like(u)
            DP = torch.zeros_like(u)
        stream.synchronize()
        return u, v, w, p, DP

    def _admit(self, req, now, stream=None):
        nbytes = footprint_bytes(req.n, self.prec)
        if nbytes > self._free(self._used):
            return None
        n = req.n
        sp = (2 * math.pi / n,) * 3
        own = stream is None
        stream = torch.cuda.Stream(self.device) if own else stream
        f = self._fields(req, stream)
        if self.batched:
            with torch.cuda.stream(stream):
                plan = Member(*f, sp, req.nu, 1.0, req.dt, min_res=self.min_res,
                              max_it=self.max_it, prec=self.prec)
        else:
            plan = StepPlan(*f, sp, req.nu, 1.0, req.dt, min_res=self.min_res,
                            max_it=self.max_it, prec=self.prec)
        self._used += nbytes
        return _Slot(req, f, plan, stream, now, nbytes)

    def _release(self, slot):
        if not self.batched:
            slot.plan.close()
        self._used -= slot.nbytes
        slot.fields = None
        slot.plan = None

    def _result(self, slot, t):
        st = slot.plan.stats()
        res = Result(slot.req.id, slot.req.n, slot.req.steps, slot.req.arrival,
                     slot.admitted, t, stats=st)
        if int(st["status"]) != 0:
            res.status = "solver-status-%d" % int(st["status"])
        if self.keep_fields:
            res.fields = tuple(f.clone() for f in slot.fields[:3])
        return res

    def _admit_arrived(self, pending, active, results, now, stream=None):
        changed = False
        while pending and pending[0].arrival <= now and len(active) < self.max_slots:
            req = pending[0]
            if footprint_bytes(req.n, self.prec) > self._capacity():
                pending.pop(0)   # can never fit: reject, do not block the queue
                results.append(Result(req.id, req.n, req.steps, req.arrival, now, now,
                                      status="rejected", error="exceeds device memory"))
                continue
            slot = self._admit(req, now, stream)
            if slot is None:
                break            # wait for memory to free up
            pending.pop(0)
            active.append(slot)
            changed = True
            self.max_active = max(self.max_active, len(active))
        return changed

    def run(self, requests, clock=None):
        """Serve ``requests`` (arrival times in seconds from now); returns the
        results in completion order."""
        if self.batched:
            return self._run_batched(requests, clock)
        return self._run_streams(requests, clock)

    def _run_batched(self, requests, clock=None):
        clock = clock or time.perf_counter
        pending = sorted(requests, key=lambda r: (r.arrival, r.id))
        active, results = [], []
        stream = torch.cuda.Stream(self.device)      # batch replays
        admit = torch.cuda.Stream(self.device)       # initial fields of admitted requests
        inflight = collections.deque()   # (event, plan, slots whose last step it ran)
        plan, dirty = None, True
        t0 = clock()
        while pending or active or inflight:
            now = clock() - t0
            # retire finished replays: their finishing requests are complete
            while inflight and inflight[0][0].query():
                _, _, done = inflight.popleft()
                t = clock() - t0
                for slot in done:
                    results.append(self._result(slot, t))
                    self._release(slot)
            if self._admit_arrived(pending, active, results, now, admit):
                dirty = True
            if active and len(inflight) < 2:
                if dirty:
                    # the old graph stays alive until its replays finish
                    plan = BatchPlan([s.plan for s in active])
                    self.rebuilds += 1
                    dirty = False
                plan.launch(1, stream=stream)
                ev = torch.cuda.Event()
                ev.record(stream)
                finishing = []
                for slot in active:
                    slot.launched += 1
                    if slot.launched >= slot.req.steps:
                        finishing.append(slot)
                for slot in finishing:
                    active.remove(slot)
                if finishing:
                    dirty = True
                inflight.append((ev, plan, finishing))
                continue
            if inflight:
                time.sleep(2e-5)
            elif pending:
                wait = pending[0].arrival - (clock() - t0)
                if wait > 0:
                    time.sleep(min(wait, 0.01))
        return results

    def _run_streams(self, requests, clock=None):
        clock = clock or time.perf_counter
        pending = sorted(requests, key=lambda r: (r.arrival, r.id))
        active, results = [], []
        t0 = clock()
        while pending or active:
            now = clock() - t0
            self._admit_arrived(pending, active, results, now)
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
                results.append(self._result(slot, clock() - t0))
                self._release(slot)
                active.remove(slot)
                progressed = True
            if not progressed:
                if active:
                    time.sleep(2e-5)
                elif pending:
                    wait = pending[0].arrival - (clock() - t0)
                    if wait > 0:
                        time.sleep(min(wait, 0.01))
        return results


def assign_requests(requests, free_bytes, prec="mixed_mg"):
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
