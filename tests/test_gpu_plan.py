"""Graph-captured steps (device-side convergence loops) reproduce the
host-driven pf_forward_step: bit for bit in FP64, and to the mixed-precision
tolerance in the mixed form; the per-step statistics match the stats kernel."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec,shape", [("fp64", (32, 32, 32)), ("fp64", (24, 20, 36)),
                                        ("mixed", (32, 32, 32)), ("mixed_mg", (32, 32, 32)),
                                        ("mixed_mg", (24, 20, 36))])
def test_plan_matches_forward_step(prec, shape):
    import pyflow_b200.initial as ic
    import pyflow_b200.ops as ops
    from pyflow_b200.plan import StepPlan
    sp = tuple(2 * np.pi / n for n in shape)
    f0 = [torch.tensor(a, device="cuda") for a in ic.spectral_velocity(shape, k0=4.0, seed=5)]
    nu, dt, steps = 0.01, 0.005, 4
    a = [t.clone() for t in f0] + [torch.zeros_like(f0[0]), torch.zeros_like(f0[0])]
    infos = []
    for _ in range(steps):
        # the mixed plans start each solve from the previous DP: so does the
        # host-driven step with warm=True
        info = ops.forward_step(*a, sp, nu, 1.0, dt, min_res=1e-10, max_it=5000, prec=prec,
                                warm=prec != "fp64")
        infos.append(info.iterations)
    b = [t.clone() for t in f0] + [torch.zeros_like(f0[0]), torch.zeros_like(f0[0])]
    plan = StepPlan(*b, sp, nu, 1.0, dt, min_res=1e-10, max_it=5000, prec=prec)
    plan.launch(steps)
    torch.cuda.synchronize()
    st = plan.stats()
    plan.close()
    assert st["status"] == 0 and st["max_res"] <= 1e-10
    if prec == "fp64":
        for x, y in zip(a[:4], b[:4]):
            assert torch.equal(x, y)
        assert int(st["iterations"]) == infos[-1]
    else:
        for x, y in zip(a[:3], b[:3]):
            assert (x - y).abs().max().item() <= 1e-12 * y.abs().max().item()
        assert int(st["iterations"]) == infos[-1]
    ref = ops.stats(*b[:3], sp).cpu().numpy()
    np.testing.assert_allclose([st["max_u"], st["max_v"], st["max_w"], st["tke"], st["max_div"]],
                               ref, rtol=1e-14, atol=1e-18)


def test_plan_mixed_fp64_fallback_matches_host_solve():
    """Unpreconditioned FP32 passes stall at 256^3 (their matvec's relative
    rounding error on the smoothest modes reaches the inner tolerance); the
    host-driven solve then switches to FP64 passes, and the captured step
    takes the same branch (an IF node on a device flag): both converge to the
    reference's tolerance with the same iteration count and the same
    velocity."""
    import pyflow_b200.initial as ic
    import pyflow_b200.ops as ops
    from pyflow_b200.plan import StepPlan
    shape = (256, 256, 256)
    sp = tuple(2 * np.pi / n for n in shape)
    f0 = [t.contiguous() for t in ic.spectral_velocity_device(shape, k0=4.0, seed=6)]
    a = [t.clone() for t in f0] + [torch.zeros_like(f0[0]), torch.zeros_like(f0[0])]
    info = ops.forward_step(*a, sp, 0.0025, 1.0, 0.00125, min_res=1e-10, max_it=20000,
                            prec="mixed")
    b = [t.clone() for t in f0] + [torch.zeros_like(f0[0]), torch.zeros_like(f0[0])]
    plan = StepPlan(*b, sp, 0.0025, 1.0, 0.00125, min_res=1e-10, max_it=20000, prec="mixed")
    plan.launch(1)
    torch.cuda.synchronize()
    st = plan.stats()
    plan.close()
    assert info.status == 0 and info.max_res <= 1e-10
    assert st["status"] == 0 and st["max_res"] <= 1e-10, st
    assert int(st["iterations"]) == info.iterations
    for x, y in zip(a[:3], b[:3]):
        assert (x - y).abs().max().item() <= 1e-12 * y.abs().max().item()


def test_plans_run_concurrently_on_streams():
    """Several plans on their own streams give the same results as alone."""
    import pyflow_b200.initial as ic
    from pyflow_b200.plan import StepPlan
    shapes = [(16, 16, 16), (24, 24, 24), (32, 32, 32)]
    alone, mixed = [], []
    for rep in range(2):
        plans, fields = [], []
        for i, sh in enumerate(shapes):
            sp = tuple(2 * np.pi / n for n in sh)
            f = [torch.tensor(a, device="cuda") for a in ic.spectral_velocity(sh, seed=20 + i)]
            f += [torch.zeros_like(f[0]), torch.zeros_like(f[0])]
            fields.append(f)
            plans.append(StepPlan(*f, sp, 0.02, 1.0, 0.004, min_res=1e-10, max_it=5000))
        torch.cuda.synchronize()
        if rep == 0:
            for pl in plans:
                pl.launch(3)
                torch.cuda.synchronize()
            alone = [f[0].clone() for f in fields]
        else:
            streams = [torch.cuda.Stream() for _ in plans]
            for _ in range(3):
                for pl, s in zip(plans, streams):
                    pl.launch(1, stream=s)
            torch.cuda.synchronize()
            mixed = [f[0].clone() for f in fields]
        for pl in plans:
            pl.close()
    for x, y in zip(alone, mixed):
        assert torch.equal(x, y)


@pytest.mark.parametrize("prec,nsets", [("fp64", 3), ("mixed_mg", 3), ("mixed_mg", 2)])
def test_pipeline_matches_plan(prec, nsets):
    """StepPipeline (two or three field sets, host copies on copy streams
    overlapped with the neighbouring requests' steps) returns, for each
    independent request, bitwise the state and statistics of one StepPlan
    step on that request."""
    import pyflow_b200.initial as ic
    from pyflow_b200.plan import StepPipeline, StepPlan
    shape = (24, 24, 32)
    sp = tuple(2 * np.pi / n for n in shape)
    nu, dt = 0.01, 0.005
    reqs = []
    for seed in range(5):
        u, v, w = ic.spectral_velocity(shape, k0=4.0, seed=20 + seed)
        p = np.random.default_rng(seed).standard_normal(shape)
        reqs.append([torch.tensor(a).pin_memory() for a in (u, v, w, p)])
    pipe = StepPipeline(shape, sp, nu, 1.0, dt, min_res=1e-10, max_it=5000, prec=prec,
                        nsets=nsets)
    stats = [torch.zeros(10, dtype=torch.float64).pin_memory() for _ in reqs]
    states = [[torch.zeros(shape, dtype=torch.float64).pin_memory() for _ in range(4)]
              for _ in reqs]
    for r, s_, o in zip(reqs, stats, states):
        pipe.submit(*r, s_, state_out=o)
    pipe.synchronize()
    pipe.close()
    for r, s_, o in zip(reqs, stats, states):
        f = [t.cuda() for t in r] + [torch.zeros(shape, dtype=torch.float64, device="cuda")]
        plan = StepPlan(*f, sp, nu, 1.0, dt, min_res=1e-10, max_it=5000, prec=prec)
        plan.launch(1)
        torch.cuda.synchronize()
        ref = plan.stats_dev.cpu()
        plan.close()
        for a, b in zip(o, f[:4]):
            assert torch.equal(a, b.cpu())
        # statistics of the step (the running totals 8, 9 differ by design)
        assert torch.equal(s_[:8], ref[:8])
        assert int(s_[7]) == 0


@pytest.mark.parametrize("prec", ["fp64", "mixed_mg"])
@pytest.mark.parametrize("closure", ["smagorinsky", "gradient", "mlp"])
def test_plan_sfs_matches_forward_step(prec, closure):
    """A plan with the SFS closure in its graph against the host-driven
    composition of Domain.forwardStep (src/data/domain.py:347-367): the
    closure by pf_sgs_closure (or pf_mlp_scales + pf_mlp_closure), the FP64
    addition of the molecular viscosity (Smagorinsky), the conversion to the
    mixed forms' FP32 stage type, then pf_forward_step with that visc or sfs.
    Bit for bit in FP64; the mixed form to the tolerance of
    test_plan_matches_forward_step.  The closure field the plan leaves is
    the one of its last step, bit for bit."""
    import pyflow_b200.initial as ic
    import pyflow_b200.ops as ops
    import pyflow_b200.sfsmodel_mlp as M
    from pyflow_b200.plan import StepPlan
    shape = (24, 20, 28)
    sp = tuple(2 * np.pi / n for n in shape)
    f0 = [torch.tensor(a, device="cuda") for a in ic.spectral_velocity(shape, k0=4.0, seed=9)]
    nu, dt, steps = 0.004, 0.004, 4
    coef = {"smagorinsky": (0.18 * sp[0]) ** 2, "gradient": sp[0] ** 2 / 12.0,
            "mlp": sp[0] * sp[0]}[closure]
    wpack = torch.as_tensor(M.pack(M.xavier_init(1))).cuda() if closure == "mlp" else None
    a = [t.clone() for t in f0] + [torch.zeros_like(f0[0]), torch.zeros_like(f0[0])]
    for _ in range(steps):
        if closure == "mlp":
            fld, _, _, err = M.closure(*a[:3], sp, wpack, sp[0])
            assert int(err.item()) == 0
        else:
            fld = ops.sgs_closure(closure, *a[:3], sp, coef=coef)
        if closure == "smagorinsky":
            fld = nu + fld
        if prec != "fp64":
            fld = fld.float()
        kw = {"visc": fld} if closure == "smagorinsky" else {"sfs": fld.contiguous()}
        info = ops.forward_step(*a, sp, nu, 1.0, dt, min_res=1e-10, max_it=5000, prec=prec,
                                warm=prec != "fp64", **kw)
    b = [t.clone() for t in f0] + [torch.zeros_like(f0[0]), torch.zeros_like(f0[0])]
    plan = StepPlan(*b, sp, nu, 1.0, dt, min_res=1e-10, max_it=5000, prec=prec,
                    closure=closure, coef=coef, wpack=wpack)
    plan.launch(steps)
    torch.cuda.synchronize()
    st = plan.stats()
    assert plan.cfield.dtype == fld.dtype and torch.equal(plan.cfield, fld)
    if closure == "mlp":
        assert int(plan.err.item()) == 0
    plan.close()
    assert st["status"] == 0 and st["max_res"] <= 1e-10
    assert int(st["iterations"]) == info.iterations
    if prec == "fp64":
        for x, y in zip(a[:4], b[:4]):
            assert torch.equal(x, y)
    else:
        for x, y in zip(a[:3], b[:3]):
            assert (x - y).abs().max().item() <= 1e-12 * y.abs().max().item()
    # the closure acted: the step differs from the one without it
    c = [t.clone() for t in f0] + [torch.zeros_like(f0[0]), torch.zeros_like(f0[0])]
    for _ in range(steps):
        ops.forward_step(*c, sp, nu, 1.0, dt, min_res=1e-10, max_it=5000, prec=prec,
                         warm=prec != "fp64")
    assert (c[0] - b[0]).abs().max().item() > 1e-9
