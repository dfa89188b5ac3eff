"""Benchmark: cell-steps/s of the RK4 + pressure-Poisson time step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--workload dns128|dns512] [--prec mixed|fp64]

A "step" is one Domain.forwardStep (src/data/domain.py:342-402): staggered RK4
predictor, divergence, BiCGStab pressure solve to max-norm relative residual
1e-10, projection.  Workload dns128 is the 128^3 decaying-turbulence DNS
(seeded k^4 exp(-2 (k/k0)^2) spectrum, k0 = 4, urms = 1, nu = 0.005,
dt = 0.0025); dns512 is the 512^3 DNS (k0 = 8, nu = 0.0012, dt = 0.001).
Inputs are synthetic (the seeded spectral field); the per-step working set
(~0.3 GB at 128^3, ~17 GB at 512^3) exceeds the 126 MB L2, so no explicit
flush is done between steps.

Under torchrun (N > 1) every rank advances its own independent replica (a
single solve of this size does not shard: "replicas only"); value is the sum of
all ranks' cell-steps over the max-over-ranks device time.

--impl reference times the reference algorithm's CPU restatement
(oracle/liboracle.so, FP64, OpenMP on all host cores) on the same workload.
"""
import argparse
import ctypes
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
    "dns512": dict(n=512, k0=8.0, nu=0.0012, dt=0.001, seed=0),
}
METRIC = "cell-steps/s (RK4+Poisson)"
TOL = 1e-10
MAX_IT = 20000


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="dns128", choices=sorted(WORKLOADS))
    ap.add_argument("--prec", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--no-fp64-arm", action="store_true",
                    help="skip the plain-FP64 comparison measurement")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-sample-steps", type=int, default=1)
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class Clocks:
    """Samples SM clocks and throttle reasons with nvidia-smi while running."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.lines = []
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                 "sw_power_cap"]
        for l in getattr(self, "lines", []):
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
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def make_fields(wl, device=None):
    """Seeded spectral initial field as float64 numpy arrays (host FFTs up to
    256^3, device FFTs above)."""
    import pyflow_b200.initial as ic
    n = wl["n"]
    if n > 256 and device is not None:
        f = ic.spectral_velocity_device((n, n, n), k0=wl["k0"], urms=1.0,
                                        seed=wl["seed"], device=device)
        out = tuple(a.cpu().numpy() for a in f)
        del f
        import torch
        torch.cuda.empty_cache()
        return out
    u, v, w = ic.spectral_velocity((n, n, n), k0=wl["k0"], urms=1.0,
                                   seed=wl["seed"])
    return u, v, w


def cpu_baseline(wl, u0, v0, w0, steps):
    """The oracle (C restatement of the reference path, FP64, OpenMP on all
    host cores) timed on a bounded sample of the workload."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle as O
    n = wl["n"]
    sp = (2 * np.pi / n,) * 3
    u, v, w, p = u0.copy(), v0.copy(), w0.copy(), np.zeros_like(u0)
    t0 = time.perf_counter()
    its = []
    for _ in range(steps):
        u, v, w, p, DP, r, it = O.forward_step(sp, u, v, w, p, wl["nu"], 1.0,
                                               wl["dt"], min_res=TOL,
                                               max_it=MAX_IT)
        its.append(it)
    el = time.perf_counter() - t0
    return {"value": n ** 3 * steps / el, "unit": "cell-steps/s",
            "cores": os.cpu_count(), "kind": "port",
            "sample": "%d FP64 step(s) of the %d^3 workload from the same "
                      "initial field (%s BiCGStab iterations)" % (steps, n, its),
            "seconds": el}


def run_reference(a):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    wl = WORKLOADS[a.workload]
    u0, v0, w0 = make_fields(wl)
    n = wl["n"]
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle as O
    sp = (2 * np.pi / n,) * 3
    u, v, w, p = u0.copy(), v0.copy(), w0.copy(), np.zeros_like(u0)
    budget = 240.0  # seconds of CPU work at most
    t_start = time.perf_counter()
    for _ in range(max(0, min(a.warmup, 1))):
        u, v, w, p, DP, r, it = O.forward_step(sp, u, v, w, p, wl["nu"], 1.0,
                                               wl["dt"], min_res=TOL,
                                               max_it=MAX_IT)
    t0 = time.perf_counter()
    done = 0
    its = []
    for _ in range(a.steps):
        u, v, w, p, DP, r, it = O.forward_step(sp, u, v, w, p, wl["nu"], 1.0,
                                               wl["dt"], min_res=TOL,
                                               max_it=MAX_IT)
        its.append(it)
        done += 1
        if time.perf_counter() - t_start > budget:
            break
    el = time.perf_counter() - t0
    val = n ** 3 * done / el
    line = {"impl": "reference", "metric": METRIC, "value": val,
            "unit": "cell-steps/s", "n_gpus": a.gpus, "steps": done,
            "warmup": min(a.warmup, 1), "ms_per_step": 1e3 * el / done,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic",
            "config": {"workload": a.workload, "grid": [n, n, n],
                       "nu": wl["nu"], "dt": wl["dt"], "tol": TOL,
                       "solver": "bicgstab", "advancer": "RK4"},
            "cpu_baseline": {"value": val, "unit": "cell-steps/s",
                             "cores": os.cpu_count(), "kind": "port",
                             "sample": "%d FP64 step(s) of the %d^3 workload "
                                       "(BiCGStab iterations %s)" % (done, n, its)},
            "e2e": {"value": val, "unit": "cell-steps/s",
                    "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_b200(a):
    import torch
    import torch.distributed as dist
    import pyflow_b200.ops as ops
    import pyflow_b200.profiling as prof

    rank, world, local = dist_env()
    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    dev = torch.device("cuda", local if world > 1 else 0)
    torch.cuda.set_device(dev)
    wl = WORKLOADS[a.workload]
    n = wl["n"]
    sp = (2 * np.pi / n,) * 3
    u0, v0, w0 = make_fields(wl, dev)

    def fresh():
        f = [torch.tensor(x, device=dev) for x in (u0, v0, w0)]
        f.append(torch.zeros_like(f[0]))
        f.append(torch.zeros_like(f[0]))
        return f

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)

    def timed(prec, steps, warmup):
        u, v, w, p, DP = fresh()
        for _ in range(warmup):
            ops.forward_step(u, v, w, p, DP, sp, wl["nu"], 1.0, wl["dt"],
                             min_res=TOL, max_it=MAX_IT, prec=prec)
        barrier()
        st = torch.cuda.current_stream(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        infos = []
        for _ in range(steps):
            info = ops.forward_step(u, v, w, p, DP, sp, wl["nu"], 1.0, wl["dt"],
                                    min_res=TOL, max_it=MAX_IT, prec=prec)
            infos.append((info.iterations, info.outer, info.max_res, info.status))
        e1.record(st)
        barrier()
        ms = e0.elapsed_time(e1)
        if world > 1:
            t = torch.tensor([ms], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        return ms, infos, (u, v, w)

    with Clocks(dev.index) as clk:
        ms, infos, fields = timed(a.prec, a.steps, a.warmup)
    clocks = clk.summary()
    value = world * n ** 3 * a.steps / (ms / 1e3)
    its = [i[0] for i in infos]

    # plain FP64 path on the same workload, and the mixed-vs-FP64 error
    fp64 = None
    if a.prec == "mixed" and not a.no_fp64_arm:
        ms64, inf64, f64 = timed("fp64", a.steps, a.warmup)
        err = max(float((x - y).abs().max() / y.abs().max())
                  for x, y in zip(fields, f64))
        fp64 = {"value": world * n ** 3 * a.steps / (ms64 / 1e3),
                "ms_per_step": ms64 / a.steps,
                "iterations_per_step": [i[0] for i in inf64],
                "mixed_rel_velocity_err": err}

    # per-kernel device time with CUDA events on the launching stream
    prof.enable(True)
    u, v, w, p, DP = fresh()
    for _ in range(max(1, min(a.steps, 2))):
        ops.forward_step(u, v, w, p, DP, sp, wl["nu"], 1.0, wl["dt"],
                         min_res=TOL, max_it=MAX_IT, prec=a.prec)
    torch.cuda.synchronize(dev)
    ktimes = prof.read()
    prof.enable(False)
    roof = prof.roofline(ktimes, n ** 3, a.prec)

    # end to end through the public API with pinned host buffers: each step
    # copies its input state in and reads the monitor statistics back
    hosts = [torch.tensor(x).pin_memory() for x in (u0, v0, w0)]
    hp = torch.zeros_like(hosts[0]).pin_memory()
    u, v, w, p, DP = fresh()
    out_h = torch.zeros(5, dtype=torch.float64).pin_memory()
    barrier()
    st = torch.cuda.current_stream(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2e_steps = max(1, min(a.steps, 3))
    e0.record(st)
    for _ in range(e2e_steps):
        for d_, h_ in zip((u, v, w, p), hosts + [hp]):
            d_.copy_(h_, non_blocking=True)
        ops.forward_step(u, v, w, p, DP, sp, wl["nu"], 1.0, wl["dt"],
                         min_res=TOL, max_it=MAX_IT, prec=a.prec)
        out_h.copy_(ops.stats(u, v, w, sp), non_blocking=True)
    e1.record(st)
    barrier()
    ms_e2e = e0.elapsed_time(e1)
    if world > 1:
        t = torch.tensor([ms_e2e], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_e2e = float(t.item())
    e2e = {"value": world * n ** 3 * e2e_steps / (ms_e2e / 1e3),
           "unit": "cell-steps/s", "h2d_bytes_per_step": 4 * 8 * n ** 3,
           "d2h_bytes_per_step": 5 * 8, "steps": e2e_steps}

    cpu = None
    if rank == 0 and not a.no_cpu_baseline:
        cpu = cpu_baseline(wl, u0, v0, w0, a.cpu_sample_steps)

    launches = sum(k["launches"] for k in ktimes.values())
    per_step_launches = launches / max(1, min(a.steps, 2))
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "cell-steps/s",
            "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": ms / a.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f32+f64" if a.prec == "mixed" else "f64",
            "data": "synthetic",
            "config": {"workload": a.workload, "grid": [n, n, n],
                       "k0": wl["k0"], "nu": wl["nu"], "dt": wl["dt"],
                       "tol": TOL, "solver": "bicgstab", "advancer": "RK4",
                       "precision": a.prec,
                       "parallelism": "replicas" if world > 1 else "single",
                       "l2": "working set > L2, no flush"},
            "iterations_per_step": its,
            "outer_per_step": [i[1] for i in infos],
            "max_res_per_step": [i[2] for i in infos],
            "fp64_arm": fp64,
            "roofline": roof,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": int(round(per_step_launches * a.steps)),
            "clocks": clocks,
            "kernels": {k: {"launches": v["launches"], "ms": v["ms"]}
                        for k, v in ktimes.items()},
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
