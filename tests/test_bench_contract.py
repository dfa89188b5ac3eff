"""bench.py's contract on the host: the reference arm (the oracle timed on the
host cores, no GPU needed) prints one JSON line with the benchmark's keys on
the GPU arm's metric and workload; its bounded per-step sample; the
one-process-per-GPU launcher and the max-over-ranks timing (gloo, world size
2)."""
import json
import os
import subprocess
import sys

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, REPO)
import bench  # noqa: E402


def _ref_line(args, timeout=600):
    r = subprocess.run([sys.executable, os.path.join(REPO, "bench.py"), "--impl", "reference"]
                       + args, cwd=REPO, capture_output=True, text=True, timeout=timeout)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout
    return json.loads(lines[0])


def _check_line(d, workload, steps):
    wl = bench.WORKLOADS[workload]
    n = wl["n"]
    assert d["impl"] == "reference"
    assert d["metric"] == bench.METRIC and d["unit"] == "cell-steps/s"
    assert d["value"] > 0 and d["higher_is_better"] is True
    assert d["steps"] == steps and d["n_gpus"] >= 1 and d["scaling"] == "weak"
    assert abs(d["ms_per_step"] - 1e3 * n ** 3 / d["value"]) <= 1e-6 * d["ms_per_step"]
    a = bench.parse(["--workload", workload])
    assert d["config"] == json.loads(json.dumps(bench.config(a, wl)))
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == d["value"]
    assert "%d^3" % n in cb["sample"]
    e = d["e2e"]
    assert e["value"] == d["value"] and e["unit"] == d["unit"]
    assert e["h2d_bytes_per_step"] == 0 and e["d2h_bytes_per_step"] == 0


def test_reference_arm_json_line():
    d = _ref_line(["--workload", "dns64", "--steps", "1", "--warmup", "0",
                   "--cpu-budget", "1"])
    _check_line(d, "dns64", 1)
    assert "whole FP64 step" in d["cpu_baseline"]["sample"]


def test_reference_arm_bounded_sample():
    d = _ref_line(["--workload", "dns64", "--steps", "1", "--warmup", "0", "--ref-sample"])
    _check_line(d, "dns64", 1)
    assert "bounded sample" in d["cpu_baseline"]["sample"]
    assert "%g iterations" % bench.WORKLOADS["dns64"]["fp64_its"] in d["cpu_baseline"]["sample"]


def test_default_workload_is_the_512_cube():
    a = bench.parse([])
    assert a.workload == "dns512" and bench.WORKLOADS["dns512"]["steps"] == 50
    assert a.gpus == 1 and a.warmup >= 3


def test_relaunch_command_runs_one_rank_per_gpu():
    cmd = bench.relaunch_command(["--gpus", "4", "--steps", "2"], 4, 29999)
    i = cmd.index("torch.distributed.run")
    assert cmd[i + 1:i + 9] == ["--nnodes=1", "--nproc-per-node", "4", "--master-addr",
                                "127.0.0.1", "--master-port", "29999",
                                os.path.join(REPO, "bench.py")]
    assert cmd[-4:] == ["--gpus", "4", "--steps", "2"]


def test_launcher_two_ranks_reference_arm():
    """--gpus 2 outside torchrun starts two ranks; rank 0 alone prints the
    reference arm's line and both exit 0."""
    env = {k: v for k, v in os.environ.items()
           if k not in ("WORLD_SIZE", "RANK", "LOCAL_RANK", "MASTER_ADDR", "MASTER_PORT")}
    r = subprocess.run([sys.executable, os.path.join(REPO, "bench.py"), "--impl", "reference",
                        "--gpus", "2", "--workload", "dns64", "--steps", "1", "--warmup", "0",
                        "--cpu-budget", "1"], cwd=REPO, capture_output=True, text=True,
                       timeout=600, env=env)
    assert r.returncode == 0, r.stderr[-3000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout
    assert json.loads(lines[0])["n_gpus"] == 2


def _max_worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms = bench.max_over_ranks(torch, dist, 10.0 * (rank + 1), torch.device("cpu"), world)
        q.put((rank, ms))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_max_over_ranks_gloo_world_size_2():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = bench.free_port()
    ps = [ctx.Process(target=_max_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(90)
        assert p.exitcode == 0
    got = dict(q.get(timeout=5) for _ in range(2))
    assert got == {0: 20.0, 1: 20.0}
