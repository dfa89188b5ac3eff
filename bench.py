"""Benchmark: cell-steps/s of the RK4 + pressure-Poisson time step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--workload dns128|dns256|dns512|serve] [--prec mixed|fp64]

A "step" is one Domain.forwardStep (src/data/domain.py:342-402): staggered RK4
predictor, divergence, BiCGStab pressure solve to max-norm relative residual
1e-10, projection -- replayed as one captured CUDA graph per step (device-side
convergence loops, no host synchronisation inside the timed region).

Precision (--prec): mixed_mg (default) runs the fluxes, RK4 stages and the
Krylov vectors in FP32 with FP64 residuals, inner products and refinement, the
FP32 passes preconditioned by a geometric multigrid V-cycle; mixed is the same
without the preconditioner; fp64 is the reference's algorithm in FP64.  The
mixed forms also time the fp64 form from the same field and report the
relative velocity difference.

Workloads (synthetic inputs: the seeded k^4 exp(-2 (k/k0)^2) spectral field,
urms = 1, in place of the reference's DNS restart data):
  dns128  128^3 decaying turbulence, k0 = 4, nu = 0.005, dt = 0.0025 (default)
  dns256  256^3, k0 = 4, nu = 0.0025, dt = 0.00125 (profiling size)
  dns512  512^3, k0 = 8, nu = 0.0012, dt = 0.001
  serve   request stream of 32..192^3 solves (50 steps each, nu = 0.02*32/N)
          with Poisson arrivals at 80 % of the measured capacity; reports
          p50/p99 latency and aggregate cell-steps/s
The per-step working set (~0.3 GB at 128^3) exceeds the 126 MB L2, so no
explicit flush is done between steps.

Under torchrun (N > 1) every rank advances its own independent replica (a
single solve of this size does not shard: "replicas only"); value is the sum of
all ranks' cell-steps over the max-over-ranks device time.

--impl reference times the reference algorithm's CPU restatement
(oracle/liboracle.so, FP64, OpenMP on all host cores) on the same workload.
"""
import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

WORKLOADS = {
    "dns128": dict(n=128, k0=4.0, nu=0.005, dt=0.0025, seed=0),
    "dns256": dict(n=256, k0=4.0, nu=0.0025, dt=0.00125, seed=0),
    "dns512": dict(n=512, k0=8.0, nu=0.0012, dt=0.001, seed=0),
}
METRIC = "cell-steps/s (RK4+Poisson)"
TOL = 1e-10
MAX_IT = 20000


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="dns128",
                    choices=sorted(WORKLOADS) + ["serve"])
    ap.add_argument("--prec", default="mixed_mg", choices=["mixed_mg", "mixed", "fp64"],
                    help="mixed_mg: FP32 refinement passes preconditioned by multigrid "
                         "(default); mixed: unpreconditioned FP32 passes; fp64: the "
                         "reference's FP64 algorithm")
    ap.add_argument("--path", default="graph", choices=["graph", "host"],
                    help="graph: captured steps replayed (default); host: host-driven "
                         "pf_forward_step per step (same kernels, host polls the solver)")
    ap.add_argument("--no-fp64-arm", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the per-kernel, e2e and MLP measurements")
    ap.add_argument("--cpu-sample-steps", type=int, default=8,
                    help="oracle steps timed for cpu_baseline (about 10 s at 128^3)")
    ap.add_argument("--requests", type=int, default=64,
                    help="serve workload: number of requests")
    return ap.parse_args()


def dist_env():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


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
    above 256^3)."""
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


def oracle_steps(wl, u0, v0, w0, steps, budget=None):
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle as O
    n = wl["n"]
    sp = (2 * np.pi / n,) * 3
    u, v, w, p = u0.copy(), v0.copy(), w0.copy(), np.zeros_like(u0)
    t0 = time.perf_counter()
    its = []
    for _ in range(steps):
        u, v, w, p, DP, r, it = O.forward_step(sp, u, v, w, p, wl["nu"], 1.0, wl["dt"],
                                               min_res=TOL, max_it=MAX_IT)
        its.append(it)
        if budget and time.perf_counter() - t0 > budget:
            break
    return time.perf_counter() - t0, its


def run_reference(a):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    if a.workload == "serve":
        print(json.dumps({"impl": "reference", "unavailable":
                          "the reference has no serving path"}), flush=True)
        return
    wl = WORKLOADS[a.workload]
    u0, v0, w0 = make_fields(wl)
    n = wl["n"]
    if min(a.warmup, 1):
        oracle_steps(wl, u0, v0, w0, 1)
    el, its = oracle_steps(wl, u0, v0, w0, a.steps, budget=240.0)
    done = len(its)
    val = n ** 3 * done / el
    sample = ("%d FP64 step(s) of the %d^3 workload from the seeded initial field "
              "(BiCGStab iterations %s)" % (done, n, its))
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": val, "unit": "cell-steps/s",
        "n_gpus": a.gpus, "steps": done, "warmup": min(a.warmup, 1),
        "ms_per_step": 1e3 * el / done, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": a.workload, "grid": [n, n, n], "nu": wl["nu"],
                   "dt": wl["dt"], "tol": TOL, "solver": "bicgstab", "advancer": "RK4"},
        "cpu_baseline": {"value": val, "unit": "cell-steps/s", "cores": os.cpu_count(),
                         "kind": "port", "sample": sample},
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
    if path == "host":
        import pyflow_b200.ops as ops
        st = torch.cuda.current_stream(dev)
        for _ in range(warmup):
            ops.forward_step(*f, sp, wl["nu"], 1.0, wl["dt"], min_res=TOL, max_it=MAX_IT,
                             prec=prec)
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        its, info = 0, None
        e0.record(st)
        for _ in range(steps):
            info = ops.forward_step(*f, sp, wl["nu"], 1.0, wl["dt"], min_res=TOL,
                                    max_it=MAX_IT, prec=prec)
            its += info.iterations
        e1.record(st)
        barrier()
        ms = e0.elapsed_time(e1)
        if world > 1:
            t = torch.tensor([ms], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        sv = ops.stats(*f[:3], sp).cpu().tolist()
        stats = dict(zip(("max_u", "max_v", "max_w", "tke", "max_div"), sv))
        stats.update(max_res=info.max_res, iterations=info.iterations, status=info.status,
                     total_iterations=its, steps=steps)
        return ms, stats, f
    plan = StepPlan(*f, sp, wl["nu"], 1.0, wl["dt"], min_res=TOL, max_it=MAX_IT, prec=prec)
    st = torch.cuda.current_stream(dev)
    plan.launch(warmup, stream=st)
    barrier()
    plan.reset_counters()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    plan.launch(steps, stream=st)
    e1.record(st)
    barrier()
    ms = e0.elapsed_time(e1)
    if world > 1:
        t = torch.tensor([ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    stats = plan.stats()
    plan.close()
    return ms, stats, f


def mlp_measurement(torch, dev):
    """Tensor-core MLP closure throughput (FLOPs of the three layers as padded
    on the tensor cores: 2*(16*128 + 128*128 + 128*16) per cell)."""
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
        flops = 2.0 * (16 * 128 + 128 * 128 + 128 * 16) * n ** 3
        ms = kt["ms"] / kt["launches"]
        out["%d^3" % n] = {"ms": ms, "tflops": flops / (ms * 1e-3) / 1e12}
        del u, v, w, res
    return out


def run_serve(a, torch, dev):
    import pyflow_b200.serving as S
    sizes = (32, 48, 64, 96, 128, 192)
    # capacity: run one request of each size alone (50 steps)
    srv = S.Server(max_slots=8, prec=a.prec, device=dev)
    cal = [S.Request(id=i, n=n, seed=999000 + i, nu=0.02 * 32 / n,
                     dt=0.3 * (2 * np.pi / n) / 4.0, steps=50) for i, n in enumerate(sizes)]
    t0 = time.perf_counter()
    for r in cal:
        srv.run([r])
    per_req = (time.perf_counter() - t0) / len(cal)   # mean service time of a request
    capacity = 1.0 / per_req
    reqs = S.stream_requests(a.requests, sizes=sizes, steps=50, rate=0.8 * capacity)
    srv = S.Server(max_slots=8, prec=a.prec, device=dev)
    t0 = time.perf_counter()
    res = srv.run(reqs)
    wall = time.perf_counter() - t0
    summ = S.summarize(res, wall)
    line = {"metric": "serve latency p50/p99 (s) and aggregate cell-steps/s",
            "value": summ["cell_steps_per_s"], "unit": "cell-steps/s", "n_gpus": 1,
            "steps": 50, "warmup": 0, "ms_per_step": None, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
            "data": "synthetic",
            "config": {"workload": "serve", "requests": a.requests, "sizes": list(sizes),
                       "steps_per_request": 50, "arrivals": "poisson",
                       "rate_per_s": 0.8 * capacity, "capacity_per_s": capacity,
                       "max_slots": 8, "precision": a.prec},
            "p50_latency_s": summ["p50_latency_s"], "p99_latency_s": summ["p99_latency_s"],
            "completed": summ["completed"], "max_active": srv.max_active,
            "wall_s": wall}
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
    value = world * n ** 3 * a.steps / (ms / 1e3)
    its_per_step = stats["total_iterations"] / max(1.0, stats["steps"])

    fp64 = None
    if a.prec != "fp64" and not a.no_fp64_arm:
        ms64, st64, f64 = timed_plan(torch, dev, u0, v0, w0, wl, "fp64", a.steps, a.warmup,
                                     barrier, world, dist, a.path)
        err = max(float((x - y).abs().max() / y.abs().max()) for x, y in zip(fields[:3], f64[:3]))
        fp64 = {"value": world * n ** 3 * a.steps / (ms64 / 1e3), "ms_per_step": ms64 / a.steps,
                "iterations_per_step": st64["total_iterations"] / max(1.0, st64["steps"]),
                "mixed_rel_velocity_err_vs_fp64": err,
                "note": "same %d warm-up + %d timed steps from the same field" % (a.warmup, a.steps)}
        del f64
    del fields

    roof, ktimes, e2e, mlp, cpu = None, {}, None, None, None
    if not a.no_extras:
        # per-kernel device time (CUDA events around each launch of the
        # host-driven path, which runs the same kernels as the graph)
        prof.enable(True)
        f = [torch.tensor(x, device=dev) for x in (u0, v0, w0)]
        f += [torch.zeros_like(f[0]), torch.zeros_like(f[0])]
        for _ in range(max(1, min(a.steps, 2))):
            ops.forward_step(*f, sp, wl["nu"], 1.0, wl["dt"], min_res=TOL, max_it=MAX_IT,
                             prec=a.prec)
        torch.cuda.synchronize(dev)
        ktimes = prof.read()
        prof.enable(False)
        roof = prof.roofline(ktimes, n ** 3, a.prec)
        if roof is not None:
            roof["step"] = prof.step_roofline(ktimes, n ** 3, max(1, min(a.steps, 2)),
                                              ms / a.steps)
        del f
        # end to end through the public API with pinned host buffers: every
        # step copies its input state in and reads the statistics back, the
        # copy of step k+1 overlapping the computation of step k
        # (plan.StepPipeline: two field sets, a copy stream)
        from pyflow_b200.plan import StepPipeline
        hosts = [torch.tensor(x).pin_memory() for x in (u0, v0, w0)]
        hp = torch.zeros_like(hosts[0]).pin_memory()
        pipe = StepPipeline((n, n, n), sp, wl["nu"], 1.0, wl["dt"], min_res=TOL, max_it=MAX_IT,
                            prec=a.prec, device=dev)
        outs = [torch.zeros(10, dtype=torch.float64).pin_memory() for _ in range(2)]
        st = pipe.compute
        e2e_steps = max(2, min(a.steps, 10))
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        pipe.copy.wait_event(e0)
        for k in range(e2e_steps):
            pipe.submit(*hosts, hp, outs[k & 1])
        pipe.copy.wait_stream(st)
        st.wait_stream(pipe.copy)
        e1.record(st)
        barrier()
        ms_e2e = e0.elapsed_time(e1)
        pipe.close()
        if world > 1:
            t = torch.tensor([ms_e2e], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms_e2e = float(t.item())
        e2e = {"value": world * n ** 3 * e2e_steps / (ms_e2e / 1e3), "unit": "cell-steps/s",
               "h2d_bytes_per_step": 4 * 8 * n ** 3, "d2h_bytes_per_step": 10 * 8,
               "steps": e2e_steps,
               "path": "pinned host u,v,w,p -> device (copy stream, overlapped with the previous "
                       "step); captured step; stats -> host"}
        del pipe, hosts
        torch.cuda.empty_cache()
        if rank == 0:
            mlp = mlp_measurement(torch, dev)
    if rank == 0 and not a.no_cpu_baseline:
        el, its = oracle_steps(wl, u0, v0, w0, a.cpu_sample_steps)
        cpu = {"value": n ** 3 * len(its) / el, "unit": "cell-steps/s", "cores": os.cpu_count(),
               "kind": "port",
               "sample": "%d FP64 step(s) of the %d^3 workload from the same initial field "
                         "(%s BiCGStab iterations), oracle/liboracle.so with OpenMP"
                         % (len(its), n, its), "seconds": el}
    launches_per_step = None
    if ktimes:
        launches_per_step = sum(k["launches"] for k in ktimes.values()) / max(1, min(a.steps, 2))
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "cell-steps/s", "n_gpus": world,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms / a.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32+f64" if a.prec != "fp64" else "f64", "data": "synthetic",
            "config": {"workload": a.workload, "grid": [n, n, n], "k0": wl["k0"],
                       "nu": wl["nu"], "dt": wl["dt"], "tol": TOL, "solver": "bicgstab",
                       "advancer": "RK4", "precision": a.prec,
                       "parallelism": "replicas" if world > 1 else "single",
                       "timing": ("captured-graph steps, device-side solver loops"
                                  if a.path == "graph" else "host-driven steps"),
                       "l2": "working set > L2, no flush"},
            "iterations_per_step": its_per_step,
            "last_step": {k: stats[k] for k in ("max_res", "iterations", "status", "tke", "max_div")},
            "fp64_arm": fp64, "roofline": roof, "cpu_baseline": cpu, "e2e": e2e,
            "gpu_launches": int(round(launches_per_step * a.steps)) if launches_per_step else None,
            "clocks": clocks, "mlp_tensor_core": mlp,
            "kernels": {k: {"launches": v["launches"], "ms": v["ms"]} for k, v in ktimes.items()},
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def main():
    a = parse()
    if a.impl == "reference":
        run_reference(a)
    else:
        run_b200(a)


if __name__ == "__main__":
    main()
