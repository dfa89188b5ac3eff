"""Benchmark: cell-steps/s of the RK4 + pressure-Poisson time step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--workload dns512|dns128|dns256|dns64|serve]
                    [--prec mixed_mg|mixed|fp64]

A "step" is one Domain.forwardStep (src/data/domain.py:342-402): staggered RK4
predictor, divergence, pressure solve to max-norm relative residual 1e-10,
projection -- replayed as one captured CUDA graph per step (device-side
convergence loops, no host synchronisation inside the timed region).

Precision (--prec):
  mixed_mg (default)  fluxes, RK4 stages and Krylov vectors in FP32; FP64
                      residuals, inner products and iterative refinement to the
                      reference's tolerance on the FP64 true residual; the FP32
                      passes run BiCGStab right-preconditioned by one FP32
                      geometric-multigrid V(2,2) cycle
  mixed               the same refinement with unpreconditioned FP32 BiCGStab
  fp64                the reference's algorithm (unpreconditioned BiCGStab) in FP64
The mixed forms also run the FP64 form from the same field for the
workload's full step count and report its rate and the error of the mixed
form against it (relative L2 / max-norm velocity error after the last step,
largest relative KE(t) and dissipation(t) errors, max|div u| of both).

Workloads (synthetic inputs: the seeded k^4 exp(-2 (k/k0)^2) spectral field,
urms = 1, in place of the reference's DNS restart data):
  dns512  512^3, k0 = 8, nu = 0.0012, dt = 0.001, 50 steps (default)
  dns128  128^3, k0 = 4, nu = 0.005, dt = 0.0025, 100 steps
  dns256  256^3, k0 = 4, nu = 0.0025, dt = 0.00125 (profiling size)
  dns64   64^3, k0 = 4, nu = 0.01, dt = 0.005, 20 steps (FP64 plain DNS)
  serve   only the request stream: 512 solves of 32..192^3 (50 steps each,
          nu = 0.02*32/N) with Poisson arrivals at 80 % of the measured
          capacity, batched serving; p50/p99 latency and aggregate
          cell-steps/s (the main run reports the same under "serve")
The per-step working set (> 0.3 GB) exceeds the 126 MB L2, so no explicit
flush is done between steps.

--gpus N without torchrun re-launches this script under torch.distributed.run
with N ranks.  Every rank advances its own independent replica (a single solve
of this size does not shard: "replicas only"); value is the sum of all ranks'
cell-steps over the max-over-ranks device time.

--impl reference times the reference algorithm's CPU restatement
(oracle/liboracle.so, FP64, OpenMP on all host cores) on the same workload; at
grids of 256^3 and more each step is a bounded sample (one step with the
pressure solve cut short, scaled to the reference's iteration count).
"""
import argparse
import json
import os
import socket
import subprocess
import sys
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

# fp64_its: BiCGStab iterations per step of the reference's algorithm on the
# workload (mean over the workload's steps, FP64 path on B200, which runs the
# reference's BiCGStab and stop test); used only to scale the CPU samples of
# grids too large to solve on the host within the benchmark's time.
WORKLOADS = {
    "dns512": dict(n=512, k0=8.0, nu=0.0012, dt=0.001, seed=0, steps=50, fp64_its=1284),
    "dns256": dict(n=256, k0=4.0, nu=0.0025, dt=0.00125, seed=0, steps=20, fp64_its=620),
    "dns128": dict(n=128, k0=4.0, nu=0.005, dt=0.0025, seed=0, steps=100, fp64_its=306),
    "dns64": dict(n=64, k0=4.0, nu=0.01, dt=0.005, seed=0, steps=20, fp64_its=150),
}
DEFAULT_WORKLOAD = "dns512"
METRIC = "cell-steps/s (RK4+Poisson)"
TOL = 1e-10
MAX_IT = 20000
SOLVER = {
    "mixed_mg": "bicgstab right-preconditioned by an fp32 multigrid V(2,2) cycle, "
                "inside fp64 iterative refinement started from the previous step's DP",
    "mixed": "fp32 bicgstab inside fp64 iterative refinement started from the previous "
             "step's DP",
    "fp64": "bicgstab (fp64, the reference's algorithm, DP = 0 at every solve)",
}


def parse(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD,
                    choices=sorted(WORKLOADS) + ["serve"])
    ap.add_argument("--prec", default="mixed_mg", choices=["mixed_mg", "mixed", "fp64"])
    ap.add_argument("--path", default="graph", choices=["graph", "host"],
                    help="graph: captured steps replayed (default); host: host-driven "
                         "pf_forward_step per step (same kernels, host polls the solver)")
    ap.add_argument("--accuracy-steps", type=int, default=None,
                    help="steps of the mixed-vs-FP64 comparison (default: the "
                         "workload's step count; 0 skips it)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the per-kernel, e2e and MLP measurements")
    ap.add_argument("--cpu-budget", type=float, default=25.0,
                    help="seconds of oracle work for cpu_baseline / the reference arm step")
    ap.add_argument("--ref-sample", action="store_true",
                    help="reference arm: use the bounded per-step sample at any grid size")
    ap.add_argument("--requests", type=int, default=512,
                    help="serve workload: number of requests")
    ap.add_argument("--no-serve", action="store_true",
                    help="skip the request-stream measurement in the main run")
    ap.add_argument("--no-les", action="store_true",
                    help="skip the LES training measurement (64^3 LES, 256^3 DNS targets)")
    return ap.parse_args(argv)


def dist_env():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def relaunch_command(argv, n, port):
    """torch.distributed.run command that runs this script with n ranks."""
    return ["timeout", "-k", "60", "3600", sys.executable, "-m", "torch.distributed.run",
            "--nnodes=1", "--nproc-per-node", str(n), "--master-addr", "127.0.0.1",
            "--master-port", str(port), os.path.abspath(__file__)] + list(argv)


def max_over_ranks(torch, dist, ms, device, world):
    """The largest of the ranks' times (the job's time)."""
    if world <= 1:
        return ms
    t = torch.tensor([ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def config(a, wl):
    """The workload, printed identically by both arms (how each arm computes
    it is in the line's "method")."""
    n = wl["n"]
    return {"workload": a.workload, "grid": [n, n, n], "k0": wl["k0"], "nu": wl["nu"],
            "dt": wl["dt"], "rho": 1.0, "tol": TOL, "steps_in_config": wl["steps"],
            "advancer": "RK4", "seed": wl["seed"],
            "l2": "working set > L2 (126 MB), no flush"}


def method(a, world):
    """How the GPU arm computes the workload."""
    return {"precision": a.prec, "solver": SOLVER[a.prec],
            "parallelism": "replicas" if world > 1 else "single",
            "timing": ("captured-graph steps, device-side solver loops"
                       if a.path == "graph" else "host-driven steps")}


class Clocks:
    """Samples SM clocks and throttle reasons with nvidia-smi while running."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            time.sleep(0.3)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            time.sleep(0.2)
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            f = [x.strip() for x in l.split(",")]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[0]))
                smax = float(f[1])
            except ValueError:
                continue
            for nm, val in zip(names, f[4:8]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def make_fields(wl, device=None):
    """Seeded spectral initial field as float64 numpy arrays (device FFTs
    above 256^3 when a device is given; same noise, same field)."""
    import pyflow_b200.initial as ic
    n = wl["n"]
    if n > 256 and device is not None:
        import torch
        f = ic.spectral_velocity_device((n, n, n), k0=wl["k0"], urms=1.0,
                                        seed=wl["seed"], device=device)
        out = tuple(a.cpu().numpy() for a in f)
        del f
        torch.cuda.empty_cache()
        return out
    return ic.spectral_velocity((n, n, n), k0=wl["k0"], urms=1.0, seed=wl["seed"])


def _oracle():
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle as O
    return O


def oracle_full_steps(wl, u0, v0, w0, budget):
    """Whole oracle steps from the initial field until ``budget`` seconds
    pass (at least one); returns (seconds, iterations per step)."""
    O = _oracle()
    n = wl["n"]
    sp = (2 * np.pi / n,) * 3
    u, v, w, p = u0.copy(), v0.copy(), w0.copy(), np.zeros_like(u0)
    t0 = time.perf_counter()
    its = []
    while True:
        u, v, w, p, DP, r, it = O.forward_step(sp, u, v, w, p, wl["nu"], 1.0, wl["dt"],
                                               min_res=TOL, max_it=MAX_IT)
        its.append(it)
        if time.perf_counter() - t0 > budget:
            break
    return time.perf_counter() - t0, its


def oracle_sampled_step(wl, u0, v0, w0, its_ref, m=(4, 24)):
    """Bounded sample of one oracle step: the step run twice from the initial
    field with the pressure solve cut at m[0] and m[1] BiCGStab iterations;
    the difference gives the time per iteration, the rest the predictor,
    divergence and projection; the step's time is scaled to ``its_ref``
    iterations.  Returns (seconds per step, description)."""
    O = _oracle()
    n = wl["n"]
    sp = (2 * np.pi / n,) * 3
    ts = []
    for mi in m:
        t0 = time.perf_counter()
        O.forward_step(sp, u0, v0, w0, np.zeros_like(u0), wl["nu"], 1.0, wl["dt"],
                       min_res=TOL, max_it=mi)
        ts.append(time.perf_counter() - t0)
    t_it = max(0.0, (ts[1] - ts[0]) / (m[1] - m[0]))
    t_fixed = max(0.0, ts[0] - m[0] * t_it)
    t_step = t_fixed + its_ref * t_it
    desc = ("bounded sample: one %d^3 step run twice from the seeded field with the "
            "BiCGStab solve cut at %d and %d iterations (%.2f s, %.2f s): %.3f s predictor"
            "+divergence+projection, %.4f s per iteration, scaled to %g iterations per step "
            "(the reference's BiCGStab on this workload)"
            % (n, m[0], m[1], ts[0], ts[1], t_fixed, t_it, its_ref))
    return t_step, desc, sum(ts)


def cpu_rate(wl, u0, v0, w0, budget, sampled, its_ref):
    """Oracle cell-steps/s on the host cores: whole steps, or the bounded
    sample.  Returns (value, sample description, seconds of work)."""
    n = wl["n"]
    if not sampled:
        el, its = oracle_full_steps(wl, u0, v0, w0, budget)
        return (n ** 3 * len(its) / el,
                "%d whole FP64 step(s) of the %d^3 workload from the seeded field "
                "(BiCGStab iterations %s)" % (len(its), n, its), el)
    t_step, desc, work = oracle_sampled_step(wl, u0, v0, w0, its_ref)
    return n ** 3 / t_step, desc, work


def run_reference(a):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    if a.workload == "serve":
        print(json.dumps({"impl": "reference", "unavailable":
                          "the reference has no serving path"}), flush=True)
        return
    wl = WORKLOADS[a.workload]
    n = wl["n"]
    dev = None
    if n > 256:
        try:
            import torch
            dev = torch.device("cuda", 0) if torch.cuda.is_available() else None
        except ImportError:
            dev = None
    u0, v0, w0 = make_fields(wl, dev)
    sampled = a.ref_sample or n >= 256
    steps = max(1, a.steps)
    warm = min(a.warmup, 1)
    if warm and not sampled:
        oracle_full_steps(wl, u0, v0, w0, 0.0)
    vals, desc = [], ""
    for _ in range(steps):
        v, desc, _ = cpu_rate(wl, u0, v0, w0, a.cpu_budget / steps, sampled, wl["fp64_its"])
        vals.append(v)
    val = float(np.mean(vals))
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": val, "unit": "cell-steps/s",
        "n_gpus": a.gpus, "steps": steps, "warmup": warm,
        "ms_per_step": 1e3 * n ** 3 / val, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": config(a, wl),
        "method": {"precision": "fp64", "solver": SOLVER["fp64"], "parallelism": "single",
                   "timing": "host wall clock of oracle steps (rank 0 only)"},
        "cpu_baseline": {"value": val, "unit": "cell-steps/s", "cores": os.cpu_count(),
                         "kind": "port", "sample": desc},
        "e2e": {"value": val, "unit": "cell-steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0}}), flush=True)


def timed_plan(torch, dev, u0, v0, w0, wl, prec, steps, warmup, barrier, world, dist,
               path="graph"):
    """K graph-replayed (or host-driven) steps bracketed by CUDA events;
    returns ms, step statistics and the fields."""
    from pyflow_b200.plan import StepPlan
    n = wl["n"]
    sp = (2 * np.pi / n,) * 3
    f = [torch.tensor(x, device=dev) for x in (u0, v0, w0)]
    f += [torch.zeros_like(f[0]), torch.zeros_like(f[0])]
    st = torch.cuda.current_stream(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if path == "host":
        import pyflow_b200.ops as ops
        warm = prec != "fp64"   # the mixed plans' initial guess: the previous DP
        for _ in range(warmup):
            ops.forward_step(*f, sp, wl["nu"], 1.0, wl["dt"], min_res=TOL, max_it=MAX_IT,
                             prec=prec, warm=warm)
        barrier()
        its, info = 0, None
        e0.record(st)
        for _ in range(steps):
            info = ops.forward_step(*f, sp, wl["nu"], 1.0, wl["dt"], min_res=TOL,
                                    max_it=MAX_IT, prec=prec, warm=warm)
            its += info.iterations
        e1.record(st)
        barrier()
        stats = dict(zip(("max_u", "max_v", "max_w", "tke", "max_div"),
                         ops.stats(*f[:3], sp).cpu().tolist()))
        stats.update(max_res=info.max_res, iterations=info.iterations, status=info.status,
                     total_iterations=its, steps=steps)
    else:
        plan = StepPlan(*f, sp, wl["nu"], 1.0, wl["dt"], min_res=TOL, max_it=MAX_IT,
                        prec=prec)
        plan.launch(warmup, stream=st)
        barrier()
        plan.reset_counters()
        e0.record(st)
        plan.launch(steps, stream=st)
        e1.record(st)
        barrier()
        stats = plan.stats()
        plan.close()
    ms = max_over_ranks(torch, dist, e0.elapsed_time(e1), dev, world)
    return ms, stats, f


def e2e_measurement(torch, dev, wl, u0, v0, w0, prec, steps, barrier, world, dist, nsets=3):
    """The metric through the public API with host buffers: every step copies
    its state (u, v, w, p, FP64) from pinned host memory to the device and the
    advanced state plus the step statistics back (plan.StepPipeline: three
    field sets; host->device and device->host copies on their own streams, so
    both copy directions and the computation overlap)."""
    from pyflow_b200.plan import StepPipeline
    n = wl["n"]
    sp = (2 * np.pi / n,) * 3
    hosts = [torch.tensor(x).pin_memory() for x in (u0, v0, w0)]
    hosts.append(torch.zeros_like(hosts[0]).pin_memory())
    outs = [[torch.empty_like(hosts[0]).pin_memory() for _ in range(4)] for _ in range(nsets)]
    stat_out = [torch.zeros(10, dtype=torch.float64).pin_memory() for _ in range(nsets)]
    pipe = StepPipeline((n, n, n), sp, wl["nu"], 1.0, wl["dt"], min_res=TOL, max_it=MAX_IT,
                        prec=prec, device=dev, nsets=nsets)
    pipe.submit(*hosts, stat_out[0], state_out=outs[0])   # warm-up
    pipe.synchronize()
    barrier()
    st = pipe.compute
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    pipe.start(e0)
    for k in range(steps):
        pipe.submit(*hosts, stat_out[k % nsets], state_out=outs[k % nsets])
    pipe.finish(st)
    e1.record(st)
    barrier()
    ms = max_over_ranks(torch, dist, e0.elapsed_time(e1), dev, world)
    pipe.close()
    # the round trip returned the state of a single step from (u0, v0, w0)
    check = float(stat_out[(steps - 1) % nsets][7])
    del hosts, outs
    return {"value": world * n ** 3 * steps / (ms / 1e3), "unit": "cell-steps/s",
            "h2d_bytes_per_step": 4 * 8 * n ** 3, "d2h_bytes_per_step": 4 * 8 * n ** 3 + 80,
            "steps": steps, "last_status": check,
            "path": ("pinned host u,v,w,p -> device (h2d stream) -> captured step -> "
                     "u,v,w,p and statistics -> pinned host (d2h stream); %d field sets, "
                     "copies of neighbouring requests overlap the computation" % nsets)}


def mlp_measurement(torch, dev):
    """Tensor-core MLP closure throughput: FLOPs of the three layers as run on
    the tensor cores (2*(16*128 + 128*128 + 128*16) per cell) and the useful
    FLOPs of the 9 -> 128 -> 128 -> 6 network (2*(9*128 + 128*128 + 128*6))."""
    import pyflow_b200.initial as ic
    import pyflow_b200.sfsmodel_mlp as M
    import pyflow_b200.profiling as prof
    out = {}
    wpack = torch.as_tensor(M.pack(M.xavier_init(1))).to(dev)
    for n in (64, 256):
        sp = (2 * np.pi / n,) * 3
        u, v, w = (t.contiguous() for t in
                   ic.spectral_velocity_device((n, n, n), k0=4.0, seed=3, device=dev))
        res = None
        for _ in range(3):
            res = M.closure(u, v, w, sp, wpack, delta=sp[0], out=res[0] if res else None)
        torch.cuda.synchronize(dev)
        prof.enable(True)
        for _ in range(5):
            res = M.closure(u, v, w, sp, wpack, delta=sp[0], out=res[0])
        torch.cuda.synchronize(dev)
        kt = prof.read().get("mlp_closure")
        prof.enable(False)
        ms = kt["ms"] / kt["launches"]
        padded = 2.0 * (16 * 128 + 128 * 128 + 128 * 16) * n ** 3
        useful = 2.0 * (9 * 128 + 128 * 128 + 128 * 6) * n ** 3
        pk, src = prof.tensor_peak()
        out["%d^3" % n] = {"ms": ms, "tflops_padded": padded / (ms * 1e-3) / 1e12,
                           "tflops_useful": useful / (ms * 1e-3) / 1e12,
                           "frac_useful_of_bf16_peak": useful / (ms * 1e-3) / 1e12 / pk,
                           "peak_tflops": pk, "peak_source": src}
        del u, v, w, res
    return out


class _UniformGeo:
    type = "uniform"

    def __init__(self, dx):
        self.dx = dx


def ml_source_measurement(torch, dev, n=64):
    """The reference's 'source' closure (273 -> 200 gated -> 18 network, one
    evaluation per RK stage) at n^3: the library's kernels (features, three
    TF32 tensor-core layers per FP32 product, closure terms) against the same
    closure as FP32 torch ops (cuBLAS GEMMs).  Useful FLOPs per cell:
    2*(3*273*200 + 2*200*200 + 200*18); executed TF32 MMA FLOPs per cell:
    3 * 2*(3*312*208 + 2*200*208 + 200*16)."""
    import pyflow_b200.initial as ic
    import pyflow_b200.sfsmodel_ML as ML
    import pyflow_b200.profiling as prof

    class _Dec:
        device = torch.device(dev)

    class _IC:
        simDt = 0.01

    torch.manual_seed(0)
    ml = ML.residual_stress(_IC(), _Dec(), _UniformGeo(2 * np.pi / n), model=ML.GatedClosureNet())
    u, v, w = (t.contiguous() for t in
               ic.spectral_velocity_device((n, n, n), k0=4.0, seed=3, device=dev))

    def timed(fn, reps):
        for _ in range(2):
            fn()
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize(dev)
        return e0.elapsed_time(e1) / reps

    ms = timed(lambda: ml.update(u, v, w), 10)
    prof.enable(True)
    for _ in range(3):
        ml.update(u, v, w)
    torch.cuda.synchronize(dev)
    kt = prof.read()
    prof.enable(False)

    def torch_path():
        with torch.no_grad():
            F = ML.features(u, v, w, ml.dx, torch.float32)
            return ML.closure_terms(ml.model(ML.network_input(F, ml.norm)), ml.dx)

    ms_torch = timed(torch_path, 5)
    useful = 2.0 * (3 * 273 * 200 + 2 * 200 * 200 + 200 * 18) * n ** 3
    executed = 3 * 2.0 * (3 * 312 * 208 + 2 * 200 * 208 + 200 * 16) * n ** 3
    out = {"grid": n, "ms": ms, "torch_fp32_ms": ms_torch,
           "tflops_useful": useful / (ms * 1e-3) / 1e12,
           "tflops_tf32_executed": executed / (ms * 1e-3) / 1e12,
           "err_flag": int(ml._err.item()),
           "kernels": {k: {"launches": v["launches"] // 3, "ms": v["ms"] / 3}
                       for k, v in kt.items() if k.startswith("mlsrc")}}
    del u, v, w, ml
    return out


def serve_measurement(a, torch, dev):
    """The request-stream workload: capacity from a burst of requests of
    every size served together, then ``a.requests`` requests with Poisson
    arrivals at 80 % of that capacity through the batched server."""
    import pyflow_b200.serving as S
    sizes = (32, 48, 64, 96, 128, 192)
    slots = 8
    burst = [S.Request(id=i, n=n, seed=999000 + i, nu=0.02 * 32 / n,
                       dt=0.3 * (2 * np.pi / n) / 4.0, steps=50)
             for i, n in enumerate(sizes * 4)]
    S.Server(max_slots=slots, prec=a.prec, device=dev).run(burst[:len(sizes)])   # warm-up
    t0 = time.perf_counter()
    S.Server(max_slots=slots, prec=a.prec, device=dev).run(burst)
    capacity = len(burst) / (time.perf_counter() - t0)
    reqs = S.stream_requests(a.requests, sizes=sizes, steps=50, rate=0.8 * capacity)
    srv = S.Server(max_slots=slots, prec=a.prec, device=dev)
    t0 = time.perf_counter()
    res = srv.run(reqs)
    wall = time.perf_counter() - t0
    summ = S.summarize(res, wall)
    return {"requests": a.requests, "completed": summ["completed"],
            "p50_latency_s": summ["p50_latency_s"], "p99_latency_s": summ["p99_latency_s"],
            "cell_steps_per_s": summ["cell_steps_per_s"], "wall_s": wall,
            "capacity_requests_per_s": capacity, "rate_requests_per_s": 0.8 * capacity,
            "sizes": list(sizes), "steps_per_request": 50, "arrivals": "poisson",
            "max_slots": slots, "max_active": srv.max_active, "batch_graphs": srv.rebuilds,
            "precision": a.prec, "solver": SOLVER[a.prec],
            "mode": "batched: one graph per active set, RK4 stages of all requests as one "
                    "grouped launch per stage, solves as parallel graph branches; "
                    "admission by live free HBM"}


def les_measurement(torch, dev, windows=3):
    """LES training at its stated size: a 64^3 LES with the tensor-core MLP
    closure (nu = 0.001, dt = 0.005), targets from a 256^3 FP64 DNS (seed 2)
    box-filtered to 64^3, 20-step windows with the loss's gradient through
    the hand-written adjoint (one checkpoint per step) and an RMSprop update
    per window.  Times the target DNS and each window (forward + backward +
    update) with CUDA events."""
    import pyflow_b200.training as T
    cfg = T.LESConfig()
    st = torch.cuda.current_stream(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    targets = T.dns_targets(cfg, device=dev)
    e1.record(st)
    torch.cuda.synchronize(dev)
    dns_s = e0.elapsed_time(e1) / 1e3
    tr = T.Trainer(cfg, targets, device=dev)
    times, losses = [], []
    for _ in range(windows):
        e0.record(st)
        losses.append(tr.step())
        e1.record(st)
        torch.cuda.synchronize(dev)
        times.append(e0.elapsed_time(e1) / 1e3)
    tr_skipped = tr.skipped
    del targets, tr
    return {"les_grid": cfg.n, "dns_grid": cfg.n * cfg.factor, "window_steps": cfg.steps,
            "windows_without_update": tr_skipped,
            "nu": cfg.nu, "dt": cfg.dt, "dns_seed": cfg.dns_seed, "mlp_seed": cfg.mlp_seed,
            "target_dns_s": dns_s, "window_s": times, "loss": losses,
            "les_cell_steps_per_s_fwd_bwd": cfg.n ** 3 * cfg.steps / float(np.median(times)),
            "note": "forward LES steps with the closure on the tensor cores, backward "
                    "through the stage-exact RK4 adjoint with recomputed stages"}


def les_plan_measurement(torch, dev, n=64, steps=20):
    """LES steps with the Smagorinsky closure (Cs = 0.18, Delta = dx) at the
    LES size of the training workload (64^3, nu = 0.001, dt = 0.005), mixed
    multigrid form: the closure inside the step graph (pf_step_plan_create_sfs)
    against the host-driven composition of Domain.forwardStep (closure,
    viscosity field, synchronous pf_forward_step), both from the same field,
    CUDA events around the same number of steps."""
    import pyflow_b200.ops as ops
    from pyflow_b200.plan import StepPlan
    u0, v0, w0 = (torch.tensor(x, device=dev)
                  for x in make_fields({"n": n, "k0": 4.0, "seed": 1}))
    sp = (2 * np.pi / n,) * 3
    nu, dt = 0.001, 0.005
    coef = (0.18 * sp[0]) ** 2
    st = torch.cuda.current_stream(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f = [u0.clone(), v0.clone(), w0.clone(), torch.zeros_like(u0), torch.zeros_like(u0)]
    plan = StepPlan(*f, sp, nu, 1.0, dt, min_res=TOL, max_it=MAX_IT, prec="mixed_mg",
                    closure="smagorinsky", coef=coef)
    plan.launch(3, stream=st)
    plan.reset_counters()
    torch.cuda.synchronize(dev)
    e0.record(st)
    plan.launch(steps, stream=st)
    e1.record(st)
    torch.cuda.synchronize(dev)
    graph_ms = e0.elapsed_time(e1) / steps
    its = plan.stats()["total_iterations"] / steps
    plan.close()
    g = [u0.clone(), v0.clone(), w0.clone(), torch.zeros_like(u0), torch.zeros_like(u0)]

    def host_step():
        visc = (nu + ops.sgs_closure("smagorinsky", *g[:3], sp, coef=coef)).float()
        ops.forward_step(*g, sp, nu, 1.0, dt, min_res=TOL, max_it=MAX_IT, prec="mixed_mg",
                         warm=True, visc=visc)

    for _ in range(3):
        host_step()
    torch.cuda.synchronize(dev)
    e0.record(st)
    for _ in range(steps):
        host_step()
    e1.record(st)
    torch.cuda.synchronize(dev)
    host_ms = e0.elapsed_time(e1) / steps
    del f, g, u0, v0, w0
    return {"grid": n, "closure": "smagorinsky", "prec": "mixed_mg", "steps": steps,
            "graph_ms_per_step": graph_ms, "host_driven_ms_per_step": host_ms,
            "iterations_per_step": its,
            "graph_cell_steps_per_s": n ** 3 / (graph_ms / 1e3)}


def slab_measurement(torch, dev, n=256, steps=2):
    """The x-slab decomposition on this one GPU (slab.LocalSlabs: the ranks'
    slabs in one process, exchanges as device copies): FP64 steps of the
    256^3 decaying-turbulence field (k0 = 4, nu = 0.005, dt = 0.0025) on one
    and on two slabs, CUDA events around the same number of steps, and the
    per-kernel roofline of the solve on one slab (launch timings of one more
    step; algorithmic bytes per interior cell from profiling.bytes_per_cell).
    Multi-GPU runs are not measured here."""
    import pyflow_b200.profiling as prof
    from pyflow_b200.slab import LocalSlabs, SlabDomain
    f0 = [torch.tensor(x, device=dev) for x in make_fields({"n": n, "k0": 4.0, "seed": 1})]
    sp = (2 * np.pi / n,) * 3
    st = torch.cuda.current_stream(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    out = {"grid": n, "prec": "fp64", "steps": steps, "transport": "LocalSlabs (one GPU)"}
    import pyflow_b200.ops as ops
    a = [t.clone() for t in f0] + [torch.zeros_like(f0[0]), torch.zeros_like(f0[0])]
    ops.forward_step(*a, sp, 0.005, 1.0, 0.0025, min_res=TOL, max_it=MAX_IT)
    torch.cuda.synchronize(dev)
    e0.record(st)
    its = sum(ops.forward_step(*a, sp, 0.005, 1.0, 0.0025, min_res=TOL, max_it=MAX_IT).iterations
              for _ in range(steps))
    e1.record(st)
    torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1) / steps
    out["single_box"] = {"ms_per_step": ms, "iterations_per_step": its / steps,
                         "ms_per_iteration": ms / max(1.0, its / steps)}
    del a
    for R in (1, 2):
        D = SlabDomain((n, n, n), sp, 0.005, 1.0, 0.0025, LocalSlabs(R), min_res=TOL,
                       max_it=MAX_IT, poll=8)
        D.set_state(*f0)
        D.forward_step()
        torch.cuda.synchronize(dev)
        e0.record(st)
        its = sum(D.forward_step().iterations for _ in range(steps))
        e1.record(st)
        torch.cuda.synchronize(dev)
        ms = e0.elapsed_time(e1) / steps
        out["slabs_%d" % R] = {"ms_per_step": ms, "iterations_per_step": its / steps,
                               "ms_per_iteration": ms / max(1.0, its / steps)}
        if R == 1:
            prof.enable(True)
            D.forward_step()
            torch.cuda.synchronize(dev)
            kt = prof.read()
            prof.enable(False)
            peak, src = prof.peaks()
            kern = {}
            for name, k in kt.items():
                b = prof.bytes_per_cell(name)
                if not name.startswith("slab_") or b is None or not k["launches"]:
                    continue
                gbs = b * n ** 3 / (k["ms"] / k["launches"] * 1e-3) / 1e9
                kern[name] = {"launches": k["launches"], "ms": k["ms"], "GB/s": gbs,
                              "frac": gbs / peak}
            out["kernels_one_slab"] = kern
            out["peak_GBs"], out["peak_source"] = peak, src
        del D
    return out


def run_serve(a, torch, dev):
    sv = serve_measurement(a, torch, dev)
    line = {"metric": "serve latency p50/p99 (s) and aggregate cell-steps/s",
            "value": sv["cell_steps_per_s"], "unit": "cell-steps/s", "n_gpus": 1,
            "steps": 50, "warmup": 0, "ms_per_step": None, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
            "data": "synthetic", "config": {"workload": "serve", "requests": a.requests},
            "serve": sv}
    print(json.dumps(line), flush=True)


def run_b200(a):
    import torch
    import torch.distributed as dist
    import pyflow_b200.ops as ops
    import pyflow_b200.profiling as prof

    rank, world, local = dist_env()
    if world > 1:
        torch.cuda.set_device(local)
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    dev = torch.device("cuda", local if world > 1 else 0)
    torch.cuda.set_device(dev)
    if a.workload == "serve":
        if rank == 0:
            run_serve(a, torch, dev)
        if world > 1:
            dist.destroy_process_group()
        return
    wl = WORKLOADS[a.workload]
    n = wl["n"]
    sp = (2 * np.pi / n,) * 3
    u0, v0, w0 = make_fields(wl, dev)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)

    with Clocks(dev.index) as clk:
        ms, stats, fields = timed_plan(torch, dev, u0, v0, w0, wl, a.prec, a.steps,
                                       a.warmup, barrier, world, dist, a.path)
    clocks = clk.summary()
    del fields
    value = world * n ** 3 * a.steps / (ms / 1e3)
    its_per_step = stats["total_iterations"] / max(1.0, stats["steps"])

    # mixed vs FP64 over the workload's step count (rank 0 of a single-GPU
    # run: the replicas would repeat the same numbers)
    fp64 = None
    acc_steps = wl["steps"] if a.accuracy_steps is None else a.accuracy_steps
    if a.prec != "fp64" and acc_steps > 0 and world == 1:
        from pyflow_b200.accuracy import compare_forms
        rep = compare_forms(u0, v0, w0, sp, wl["nu"], wl["dt"], acc_steps, prec=a.prec,
                            device=dev)
        rep.pop("per_step")
        fp64 = {"value": n ** 3 / (rep["fp64_ms_per_step"] / 1e3),
                "ms_per_step": rep["fp64_ms_per_step"],
                "iterations_per_step": rep["fp64_iterations_per_step"],
                "solver": SOLVER["fp64"],
                "errors_of_%s_vs_fp64" % a.prec: {
                    k: rep[k] for k in ("steps", "u_rel_l2", "u_rel_linf", "ke_rel_err_max",
                                        "dissipation_rel_err_max", "max_div_fp64",
                                        "max_div_mixed", "ke_decay", "mixed_status",
                                        "fp64_status")},
                "note": "%d steps of each form from the same field, per-step flow statistics "
                        "included in both times" % acc_steps}
        torch.cuda.empty_cache()

    roof, ktimes, e2e, mlp, cpu, serve, les = None, {}, None, None, None, None, None
    mlsrc = les_plan = slab = None
    prof_steps = 2
    if not a.no_extras:
        # per-kernel device time: CUDA events around each launch of the
        # host-driven path, which runs the kernels of the captured step (in
        # the mixed forms from the previous step's DP, as the plans do)
        prof.enable(True)
        f = [torch.tensor(x, device=dev) for x in (u0, v0, w0)]
        f += [torch.zeros_like(f[0]), torch.zeros_like(f[0])]
        for _ in range(prof_steps):
            ops.forward_step(*f, sp, wl["nu"], 1.0, wl["dt"], min_res=TOL, max_it=MAX_IT,
                             prec=a.prec, warm=a.prec != "fp64")
        torch.cuda.synchronize(dev)
        ktimes = prof.read()
        prof.enable(False)
        del f
        roof = prof.roofline(ktimes, n ** 3, a.prec)
        if roof is not None:
            roof["step"] = prof.step_roofline(ktimes, n ** 3, prof_steps, ms / a.steps)
            roof["kernel_times"] = ("CUDA events around every launch of %d host-driven steps "
                                    "(%.3f ms of kernel time per step against %.3f ms per "
                                    "graph-replayed step)"
                                    % (prof_steps, sum(k["ms"] for k in ktimes.values())
                                       / prof_steps, ms / a.steps))
        torch.cuda.empty_cache()
        # as many requests as the timed region has steps, so the pipeline's
        # fill and drain (one copy-in, one copy-out) weigh as in a request stream
        e2e = e2e_measurement(torch, dev, wl, u0, v0, w0, a.prec, max(3, a.steps),
                              barrier, world, dist)
        torch.cuda.empty_cache()
        if rank == 0:
            mlp = mlp_measurement(torch, dev)
            torch.cuda.empty_cache()
            mlsrc = ml_source_measurement(torch, dev)
            torch.cuda.empty_cache()
            les_plan = les_plan_measurement(torch, dev)
            torch.cuda.empty_cache()
            slab = slab_measurement(torch, dev)
            torch.cuda.empty_cache()
            if not a.no_serve and world == 1:
                serve = serve_measurement(a, torch, dev)
                torch.cuda.empty_cache()
            if not a.no_les and world == 1:
                try:
                    les = les_measurement(torch, dev)
                except RuntimeError as e:   # reported, the rest of the line stands
                    les = {"error": str(e)}
                torch.cuda.empty_cache()
    if rank == 0 and not a.no_cpu_baseline:
        its_ref = fp64["iterations_per_step"] if fp64 else wl["fp64_its"]
        val, desc, work = cpu_rate(wl, u0, v0, w0, a.cpu_budget, n >= 256, its_ref)
        cpu = {"value": val, "unit": "cell-steps/s", "cores": os.cpu_count(), "kind": "port",
               "sample": desc + "; oracle/liboracle.so (FP64, OpenMP)", "seconds": work}
    launches_per_step = None
    if ktimes:
        launches_per_step = sum(k["launches"] for k in ktimes.values()) / prof_steps
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "cell-steps/s", "n_gpus": world,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms / a.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32+f64" if a.prec != "fp64" else "f64", "data": "synthetic",
            "config": config(a, wl), "method": method(a, world),
            "iterations_per_step": its_per_step,
            "last_step": {k: stats[k] for k in ("max_res", "iterations", "status", "tke",
                                                "max_div")},
            "fp64_arm": fp64, "roofline": roof, "cpu_baseline": cpu, "e2e": e2e,
            "gpu_launches": int(round(launches_per_step * a.steps)) if launches_per_step else None,
            "clocks": clocks, "mlp_tensor_core": mlp, "ml_source_closure": mlsrc,
            "serve": serve, "les_training": les, "les_step_graph": les_plan,
            "slab_decomposition": slab,
            "kernels": {k: {"launches": v["launches"], "ms": v["ms"]} for k, v in ktimes.items()},
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def main(argv=None):
    argv = sys.argv[1:] if argv is None else argv
    a = parse(argv)
    if a.gpus > 1 and "WORLD_SIZE" not in os.environ:
        # one process per GPU: re-launch under torch.distributed.run
        sys.exit(subprocess.call(relaunch_command(argv, a.gpus, free_port())))
    if a.impl == "reference":
        run_reference(a)
    else:
        run_b200(a)


if __name__ == "__main__":
    main()
