"""Failure detection without faulting the GPU: every solver loop ends on its
own (device-side stop tests, bounded iteration counts) and reports a status
the host reads, with the CUDA context still usable afterwards.  Failures are
made on the host side: a NaN in the input, an iteration limit that is too
small, a zero right-hand side."""
import math

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

PF_OK, PF_MAXIT, PF_NONFINITE = 0, 4, 5


def _source(n=32, seed=1):
    import pyflow_b200.ops as ops
    rng = np.random.default_rng(seed)
    sp = (2 * math.pi / n,) * 3
    u, v, w = (torch.tensor(rng.standard_normal((n,) * 3), device="cuda") for _ in range(3))
    return ops.div_vel(u, v, w, sp), sp


@pytest.mark.parametrize("prec", ["fp64", "mixed", "mixed_mg"])
def test_nan_source_reports_nonfinite(prec):
    import pyflow_b200.ops as ops
    src, sp = _source()
    src[3, 4, 5] = float("nan")
    DP, p = torch.zeros_like(src), torch.zeros_like(src)
    info = ops.bicgstab_solve(src, DP, p, sp, 1.0, 0.01, 1e-10, 500, prec=prec)
    assert info.status == PF_NONFINITE
    # the context is still usable: a clean solve right after succeeds
    src2, _ = _source()
    DP.zero_(); p.zero_()
    assert ops.bicgstab_solve(src2, DP, p, sp, 1.0, 0.01, 1e-10, 5000, prec=prec).status == PF_OK


@pytest.mark.parametrize("prec", ["fp64", "mixed", "mixed_mg"])
def test_iteration_limit_reports_maxit(prec):
    import pyflow_b200.ops as ops
    src, sp = _source()
    DP, p = torch.zeros_like(src), torch.zeros_like(src)
    info = ops.bicgstab_solve(src, DP, p, sp, 1.0, 0.01, 1e-14, 3, prec=prec)
    assert info.status == PF_MAXIT
    assert info.iterations <= 3 + 1


def test_plan_with_nan_velocity_stops():
    """A captured step whose velocity holds a NaN ends its device-side loops
    and reports a non-OK status instead of spinning."""
    import pyflow_b200.initial as ic
    from pyflow_b200.plan import StepPlan
    n = 24
    sp = (2 * math.pi / n,) * 3
    f = [torch.tensor(a, device="cuda") for a in ic.spectral_velocity((n,) * 3, seed=3)]
    f[0][1, 2, 3] = float("nan")
    f += [torch.zeros_like(f[0]), torch.zeros_like(f[0])]
    for prec in ("fp64", "mixed", "mixed_mg"):
        g = [t.clone() for t in f]
        plan = StepPlan(*g, sp, 0.01, 1.0, 0.005, min_res=1e-10, max_it=500, prec=prec)
        plan.launch(2)
        torch.cuda.synchronize()
        st = plan.stats()
        plan.close()
        assert int(st["status"]) != PF_OK, (prec, st)
        assert st["iterations"] <= 500


def test_pyflow_error_carries_status():
    import pyflow_b200._lib as L
    import pyflow_b200.ops as ops
    src, sp = _source(16)
    DP = torch.zeros_like(src)
    with pytest.raises(L.PyFlowError) as e:
        # dt == 0 is rejected by the C ABI before any launch
        ops.bicgstab_solve(src, DP, torch.zeros_like(src), sp, 1.0, 0.0, 1e-10, 10)
    assert e.value.status == 1
