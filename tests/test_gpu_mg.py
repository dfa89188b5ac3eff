"""Multigrid-preconditioned mixed-precision pressure solve (PF_MIXED_MG).

The reference's BiCGStab is unpreconditioned; PF_MIXED_MG changes only how
the FP32 refinement passes reach their tolerance.  It must converge to the
same FP64 tolerance (checked on the true residual b - A DP recomputed in FP64),
give the FP64 solver's DP to the accuracy that tolerance implies, and take far
fewer iterations.  Grids that cannot be coarsened run the PF_MIXED passes."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _source(shape, seed):
    import pyflow_b200.ops as ops
    sp = tuple(2 * np.pi / n for n in shape)
    rng = np.random.default_rng(seed)
    u, v, w = (torch.tensor(rng.standard_normal(shape), device="cuda") for _ in range(3))
    return ops.div_vel(u, v, w, sp), sp


def _solve(src, sp, prec, rho=1.0, dt=0.01, tol=1e-10, max_it=20000):
    import pyflow_b200.ops as ops
    DP = torch.zeros_like(src)
    p = torch.zeros_like(src)
    info = ops.bicgstab_solve(src, DP, p, sp, rho, dt, tol, max_it, prec=prec)
    torch.cuda.synchronize()
    return DP, info


def _true_residual(src, DP, sp, rho=1.0, dt=0.01):
    import pyflow_b200.ops as ops
    vol = sp[0] * sp[1] * sp[2]
    b = (src * (rho / dt)) * (-vol)
    r = b - ops.laplace_apply(DP, sp)
    return float(r.abs().max() / b.abs().max())


@pytest.mark.parametrize("shape", [(32, 32, 32), (24, 20, 36), (64, 64, 64), (48, 64, 32)])
def test_mg_solve_matches_fp64(shape):
    src, sp = _source(shape, seed=11)
    DP64, i64 = _solve(src, sp, "fp64")
    DPmg, img = _solve(src, sp, "mixed_mg")
    assert i64.status == 0 and img.status == 0
    assert img.max_res <= 1e-10
    assert _true_residual(src, DPmg, sp) <= 1e-10
    a = DPmg - DPmg.mean()
    b = DP64 - DP64.mean()
    assert float((a - b).abs().max()) <= 1e-6 * float(b.abs().max())
    if shape[0] >= 48:
        assert img.iterations * 4 < i64.iterations, (img.iterations, i64.iterations)


def test_mg_odd_grid_runs_mixed_passes():
    """33 cannot be halved: the solve uses the unpreconditioned FP32 passes."""
    src, sp = _source((33, 20, 20), seed=3)
    DPm, im = _solve(src, sp, "mixed")
    DPg, ig = _solve(src, sp, "mixed_mg")
    assert ig.status == 0 and _true_residual(src, DPg, sp) <= 1e-10
    assert torch.equal(DPm, DPg) and im.iterations == ig.iterations


def test_mg_zero_source():
    src = torch.zeros(32, 32, 32, dtype=torch.float64, device="cuda")
    DP, info = _solve(src, (0.2,) * 3, "mixed_mg")
    assert info.status == 0 and float(DP.abs().max()) == 0.0


def test_mg_forward_steps_match_fp64():
    """Five RK4 + projection steps of a 32^3 spectral field: PF_MIXED_MG stays
    within 1e-7 (relative) of the FP64 path."""
    import pyflow_b200.initial as ic
    import pyflow_b200.ops as ops
    shape = (32, 32, 32)
    sp = (2 * np.pi / 32,) * 3
    f0 = [torch.tensor(a, device="cuda") for a in ic.spectral_velocity(shape, k0=4.0, seed=0)]
    out = {}
    for prec in ("fp64", "mixed_mg"):
        f = [t.clone() for t in f0] + [torch.zeros_like(f0[0]), torch.zeros_like(f0[0])]
        for _ in range(5):
            info = ops.forward_step(*f, sp, 0.01, 1.0, 0.005, min_res=1e-10, max_it=5000,
                                    prec=prec)
            assert info.status == 0
        out[prec] = f
    for x, y in zip(out["mixed_mg"][:3], out["fp64"][:3]):
        assert float((x - y).abs().max()) <= 1e-7 * float(y.abs().max())
    div = ops.div_vel(*out["mixed_mg"][:3], sp)
    assert float(div.abs().max()) < 1e-8


_COOP_SCRIPT = r"""
import sys, numpy as np, torch
sys.path.insert(0, {repo!r})
import pyflow_b200.ops as ops
from pyflow_b200.plan import StepPlan
import pyflow_b200.initial as ic
out = {{}}
for n in (64, 128):
    g = torch.Generator().manual_seed(n)
    src = torch.randn((n, n, n), generator=g, dtype=torch.float64).cuda()
    src -= src.mean()
    sp = (2 * np.pi / n,) * 3
    DP = torch.zeros_like(src); p = torch.zeros_like(src)
    ops.bicgstab_solve(src, DP, p, sp, 1.0, 0.01, 1e-10, 2000, prec="mixed_mg")
    torch.cuda.synchronize()
    out["solve%d" % n] = DP.cpu().numpy()
n = 128
u, v, w = (torch.tensor(a, device="cuda") for a in ic.spectral_velocity((n, n, n), seed=4))
f = [u, v, w, torch.zeros_like(u), torch.zeros_like(u)]
plan = StepPlan(*f, (2 * np.pi / n,) * 3, 0.005, 1.0, 0.0025, prec="mixed_mg")
plan.launch(3)
torch.cuda.synchronize()
plan.close()
for k, t in zip("uvwp", f[:4]):
    out["step_" + k] = t.cpu().numpy()
np.savez({path!r}, **out)
"""


def test_mg_cooperative_mid_levels_bit_identical(tmp_path):
    """The one-thread-per-cell levels as two cooperative launches per V-cycle
    (PF_MG_COOP=1) and as per-level kernels (default) give bit-identical
    solves (64^3, 128^3, host-driven) and steps (128^3, captured plan)."""
    import os
    import subprocess
    import sys
    repo = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    res = {}
    for mode in ("1", "0"):
        path = str(tmp_path / ("coop%s.npz" % mode))
        env = dict(os.environ, PF_MG_COOP=mode)
        r = subprocess.run([sys.executable, "-c", _COOP_SCRIPT.format(repo=repo, path=path)],
                           env=env, capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr[-3000:]
        res[mode] = np.load(path)
    for k in res["1"].files:
        assert np.array_equal(res["1"][k], res["0"][k]), k


def test_mg_cooperative_path_runs(monkeypatch):
    """With PF_MG_COOP=1, the host-driven mixed_mg solve at 128^3 launches the
    cooperative mid levels (two per V-cycle) and no per-level kernels of
    those levels."""
    import pyflow_b200.ops as ops
    import pyflow_b200.profiling as prof
    monkeypatch.setenv("PF_MG_COOP", "1")
    n = 128
    g = torch.Generator().manual_seed(1)
    src = torch.randn((n, n, n), generator=g, dtype=torch.float64).cuda()
    src -= src.mean()
    sp = (2 * np.pi / n,) * 3
    DP = torch.zeros_like(src)
    p = torch.zeros_like(src)
    prof.enable(True)
    info = ops.bicgstab_solve(src, DP, p, sp, 1.0, 0.01, 1e-10, 2000, prec="mixed_mg")
    torch.cuda.synchronize()
    kt = prof.read()
    prof.enable(False)
    assert info.status == 0
    assert kt.get("mg_mid_down", {}).get("launches", 0) > 0
    assert kt["mg_mid_down"]["launches"] == kt["mg_mid_up"]["launches"]
    assert "mg_smooth0_pw" not in kt and "mg_prolong_smooth_pw" not in kt
    assert _true_residual(src, DP, sp) <= 1e-10
