"""CUDA path vs the reference's golden fixtures and the CPU oracle.

FP64 elementwise operators (RHS, RK4/Euler predictors, divergence, Laplacian,
projection, Jacobi) must match the reference bit for bit.  The BiCGStab solve
matches to the reference's own round-off sensitivity (the dot products sum in a
different order): same stop criterion, iteration count within 10 %, DP within
2e-8 relative.  Mixed precision is checked against the FP64 oracle with the
tolerance stated per test.
"""
import numpy as np
import pytest
import torch

import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ops():
    import pyflow_b200.ops as ops
    return ops


def cu(a, dtype=torch.float64):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device="cuda")


def host(t):
    torch.cuda.synchronize()
    return t.detach().cpu().numpy()


def test_rhs_fp64_bitexact(ops, golden):
    g = golden("ops_12x16x20.npz")
    out = ops.rhs_ns(cu(g["u"]), cu(g["v"]), cu(g["w"]), g["spacing"],
                     float(g["mu"]), float(g["rho"]))
    assert np.array_equal(np.stack([host(t) for t in out]), g["rhs_const"])
    out = ops.rhs_ns(cu(g["u"]), cu(g["v"]), cu(g["w"]), g["spacing"], 0.0,
                     float(g["rho"]), visc=cu(g["visc"]), sfs=cu(g["sfs"]))
    assert np.array_equal(np.stack([host(t) for t in out]), g["rhs_visc_sfs"])


def test_rhs_fp32_close_to_fp64(ops, golden):
    g = golden("ops_12x16x20.npz")
    f = torch.float32
    out = ops.rhs_ns(cu(g["u"], f), cu(g["v"], f), cu(g["w"], f), g["spacing"],
                     float(g["mu"]), float(g["rho"]))
    ref = g["rhs_const"]
    err = np.abs(np.stack([host(t) for t in out]) - ref).max()
    assert err <= 1e-5 * np.abs(ref).max()


def test_div_laplace_bitexact(ops, golden):
    g = golden("ops_12x16x20.npz")
    d = ops.div_vel(cu(g["u"]), cu(g["v"]), cu(g["w"]), g["spacing"])
    assert np.array_equal(host(d), g["div"])
    b = ops.laplace_apply(cu(g["u"]), g["spacing"])
    assert np.array_equal(host(b), g["lap_u"])


@pytest.mark.parametrize("rk4,key", [(True, "rk4"), (False, "euler")])
def test_predictor_bitexact(ops, golden, rk4, key):
    g = golden("ops_12x16x20.npz")
    u, v, w = cu(g["u"]), cu(g["v"]), cu(g["w"])
    ops.predictor_step(u, v, w, g["spacing"], float(g["mu"]), float(g["rho"]),
                       float(g["dt"]), rk4=rk4)
    assert np.array_equal(np.stack([host(u), host(v), host(w)]), g[key])


def test_bicgstab_fp64_vs_reference(ops, golden):
    g = golden("ops_12x16x20.npz")
    src = cu(g["bicg_source"])
    DP = torch.zeros_like(src)
    p = cu(g["p0"])
    info = ops.bicgstab_solve(src, DP, p, g["spacing"], float(g["rho"]),
                              float(g["dt"]), 1e-10, 500)
    ref_it = int(g["bicg_iters"])
    assert info.status == 0
    assert abs(info.iterations - ref_it) <= max(2, ref_it // 10)
    assert info.max_res <= 1e-10
    scale = np.abs(g["bicg_DP"]).max()
    assert np.abs(host(DP) - g["bicg_DP"]).max() <= 2e-8 * scale
    assert np.abs(host(p) - g["bicg_p"]).max() <= 2e-8 * scale
    # the source is not modified
    assert np.array_equal(host(src), g["bicg_source"])


def test_bicgstab_deterministic(ops, golden):
    g = golden("ops_12x16x20.npz")
    outs = []
    for _ in range(2):
        src = cu(g["bicg_source"])
        DP = torch.zeros_like(src)
        p = torch.zeros_like(src)
        info = ops.bicgstab_solve(src, DP, p, g["spacing"], float(g["rho"]),
                                  float(g["dt"]), 1e-10, 500)
        outs.append((host(DP), info.iterations, info.max_res))
    assert np.array_equal(outs[0][0], outs[1][0])
    assert outs[0][1:] == outs[1][1:]


def test_vel_corr_bitexact_vs_oracle(ops, golden):
    g = golden("ops_12x16x20.npz")
    DP = g["bicg_DP"]
    scale = float(g["dt"]) / float(g["rho"])
    ref = O.vel_corr(g["spacing"], DP, scale, *g["rk4"])
    u, v, w = (cu(a) for a in g["rk4"])
    ops.vel_corr(cu(DP), scale, u, v, w, g["spacing"])
    assert np.array_equal(np.stack([host(u), host(v), host(w)]), np.stack(ref))


def test_jacobi_bitexact(ops, golden):
    g = golden("jacobi_16.npz")
    src = cu(g["source"])
    pold = torch.zeros_like(src)
    p = torch.ones_like(src)
    r = ops.jacobi_solve(src, pold, p, g["spacing"], float(g["rho"]),
                         float(g["dt"]), int(g["n_it"]))
    assert np.array_equal(host(p), g["p"])
    assert np.array_equal(host(pold), g["DP"])
    assert r == float(g["max_res"])


def _run(ops, g, prec):
    u, v, w = cu(g["u0"]), cu(g["v0"]), cu(g["w0"])
    p = torch.zeros_like(u)
    DP = torch.zeros_like(u)
    infos = []
    for s in range(int(g["steps"])):
        info = ops.forward_step(u, v, w, p, DP, g["spacing"], float(g["nu"]),
                                float(g["rho"]), float(g["dt"]), min_res=1e-10,
                                max_it=1000, prec=prec)
        infos.append((info.iterations, info.max_res, info.status))
    return u, v, w, p, infos


def test_forward_run_fp64_vs_reference(ops, golden):
    g = golden("run_32.npz")
    u, v, w, p, infos = _run(ops, g, "fp64")
    its = np.array([i[0] for i in infos])
    assert all(i[2] == 0 for i in infos)
    assert np.all(np.abs(its - g["iters"]) <= 0.1 * g["iters"])
    # BiCGStab stops at a 1e-10 max-norm relative residual and its iterates
    # depend on the dot-product summation order, so velocities agree to the
    # solver tolerance rather than bit for bit
    for a, key in ((u, "u"), (v, "v"), (w, "w")):
        ref = g[key]
        assert np.abs(host(a) - ref).max() <= 1e-9 * np.abs(ref).max()
    assert np.abs(host(p) - g["p"]).max() <= 1e-8 * np.abs(g["p"]).max()


@pytest.mark.parametrize("prec", ["mixed", "mixed_mg"])
def test_forward_run_mixed_vs_reference(ops, golden, prec):
    """Mixed precision: FP32 fluxes/stages/matvec, FP64 state, residual and
    refinement to the same 1e-10 tolerance.  Velocity within 1e-6 relative."""
    g = golden("run_32.npz")
    u, v, w, p, infos = _run(ops, g, prec)
    assert all(i[2] == 0 for i in infos), infos
    assert all(i[1] <= 1e-10 for i in infos)
    for a, key in ((u, "u"), (v, "v"), (w, "w")):
        ref = g[key]
        assert np.abs(host(a) - ref).max() <= 1e-6 * np.abs(ref).max()


def test_stats_vs_oracle(ops, golden):
    g = golden("run_32.npz")
    st = host(ops.stats(cu(g["u"]), cu(g["v"]), cu(g["w"]), g["spacing"]))
    ref = O.stats(g["spacing"], g["u"], g["v"], g["w"])
    np.testing.assert_allclose(st[:3], ref[:3], rtol=0, atol=0)
    np.testing.assert_allclose(st[3], ref[3], rtol=1e-13)
    np.testing.assert_allclose(st[4], ref[4], rtol=1e-12, atol=1e-16)


@pytest.mark.parametrize("shape", [(64, 48, 40), (33, 17, 70)])
def test_ragged_shapes_vs_oracle(ops, shape):
    """Non-multiple-of-tile shapes: RHS and predictor bit-exact, BiCGStab to
    the same tolerance, divergence-free after the projection."""
    rng = np.random.default_rng(5)
    u, v, w = (rng.standard_normal(shape) for _ in range(3))
    sp = (0.1, 0.13, 0.07)
    out = ops.rhs_ns(cu(u), cu(v), cu(w), sp, 0.02, 1.0)
    ref = O.rhs_ns(sp, u, v, w, 0.02, 1.0)
    for a, b in zip(out, ref):
        assert np.array_equal(host(a), b)
    uu, vv, ww = cu(u), cu(v), cu(w)
    p, DP = torch.zeros_like(uu), torch.zeros_like(uu)
    info = ops.forward_step(uu, vv, ww, p, DP, sp, 0.02, 1.0, 1e-3,
                            min_res=1e-10, max_it=2000)
    ru, rv, rw, rp, rDP, rres, rit = O.forward_step(
        sp, u, v, w, np.zeros(shape), 0.02, 1.0, 1e-3, min_res=1e-10,
        max_it=2000)
    assert info.status == 0 and info.max_res <= 1e-10
    assert abs(info.iterations - rit) <= max(3, rit // 10)
    for a, b in ((uu, ru), (vv, rv), (ww, rw)):
        assert np.abs(host(a) - b).max() <= 1e-8 * np.abs(b).max()
    st = host(ops.stats(uu, vv, ww, sp))
    assert st[4] <= 1e-8 * st[0] / min(sp)


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-9), ("mixed", 1e-6), ("mixed_mg", 1e-6)])
def test_run_64_twenty_steps_vs_reference(golden, prec, tol):
    """The 64^3 plain-DNS workload (seed 0, nu = 0.01, dt = 0.005, 20 RK4 steps)
    through the captured-graph path against the reference's own run."""
    import pyflow_b200.initial as ic
    from pyflow_b200.plan import StepPlan
    g = golden("run_64.npz")
    n = int(g["shape"][0])
    f = [cu(a) for a in ic.spectral_velocity((n, n, n), k0=float(g["k0"]),
                                             urms=float(g["urms"]), seed=int(g["seed"]))]
    f += [torch.zeros_like(f[0]), torch.zeros_like(f[0])]
    plan = StepPlan(*f, g["spacing"], float(g["nu"]), float(g["rho"]), float(g["dt"]),
                    min_res=1e-10, max_it=1000, prec=prec)
    its = []
    for s in range(int(g["steps"])):
        plan.launch(1)
        st = plan.stats()
        its.append(st["iterations"])
        assert st["status"] == 0 and st["max_res"] <= 1e-10
        np.testing.assert_allclose([st["max_u"], st["max_v"], st["max_w"], st["tke"]],
                                   g["stats"][s][:4], rtol=max(tol, 1e-10))
    plan.close()
    if prec == "fp64":
        assert np.all(np.abs(np.array(its) - g["iters"]) <= 0.1 * g["iters"])
    k = int(g["stride"])
    for a, key in zip(f[:3], ("u", "v", "w")):
        ref = g[key + "_sub"]
        got = host(a)[::k, ::k, ::k]
        assert np.abs(got - ref).max() <= tol * np.abs(ref).max()


@pytest.mark.parametrize("shape", [(64, 48, 40), (33, 17, 70), (6, 4, 5)])
@pytest.mark.parametrize("rk4", [True, False])
def test_predictor_tiled_bitexact_vs_oracle(ops, shape, rk4):
    """The tiled stage kernels (constant viscosity, no SFS) on shapes that are
    not tile multiples, including dimensions smaller than the tile and its
    halo: bit-exact against the oracle's RK4 / Euler predictor."""
    rng = np.random.default_rng(9)
    u, v, w = (rng.standard_normal(shape) for _ in range(3))
    sp = (0.1, 0.13, 0.07)
    uu, vv, ww = cu(u), cu(v), cu(w)
    ops.predictor_step(uu, vv, ww, sp, 0.02, 1.1, 1e-3, rk4=rk4)
    if rk4:
        ref = O.rk4_step(sp, u, v, w, 0.02, 1.1, 1e-3)
    else:
        k = O.rhs_ns(sp, u, v, w, 0.02, 1.1)
        ref = tuple(a + b * 1e-3 for a, b in zip((u, v, w), k))
    for a, b in zip((uu, vv, ww), ref):
        assert np.array_equal(host(a), b)


def test_predictor_mixed_tiled_matches_gather(ops):
    """Mixed-precision stages: the tiled kernels (constant viscosity) and the
    gather kernels (here forced by a uniform viscosity field equal to mu)
    compute the same FP32 arithmetic."""
    rng = np.random.default_rng(4)
    shape = (40, 36, 48)
    u, v, w = (rng.standard_normal(shape) for _ in range(3))
    sp = (0.1, 0.1, 0.1)
    a = [cu(x) for x in (u, v, w)]
    b = [cu(x) for x in (u, v, w)]
    ops.predictor_step(*a, sp, 0.02, 1.0, 1e-3, prec="mixed")
    visc = torch.full(shape, 0.02, dtype=torch.float32, device="cuda")
    ops.predictor_step(*b, sp, 0.02, 1.0, 1e-3, prec="mixed", visc=visc)
    for x, y in zip(a, b):
        assert float((x - y).abs().max()) <= 1e-6 * float(y.abs().max())
