"""The target-data corrector (Domain.TargetDataVelCorr, src/data/domain.py:445-468)
against the reference's own run on a random, not divergence-free target field
(tests/golden/target_12x16x20.npz): the projected target velocity, the DP of
the solve and the simulation pressure to which the reference's solve adds DP.
BiCGStab's dot products sum in a different order than torch.sum, so the
solve agrees to round-off: DP within 2e-8 and the velocities within 1e-9
(relative max norms)."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def test_target_projection_matches_reference(golden):
    from pyflow_b200.adjoint import project
    import pyflow_b200.ops as ops
    g = golden("target_12x16x20.npz")
    cu = lambda a: torch.tensor(np.ascontiguousarray(a), device="cuda")
    tgt = [cu(g[k]) for k in ("uT", "vT", "wT")]
    p, DP = cu(g["p0"]), torch.zeros_like(tgt[0])
    info = project(tgt, g["spacing"], float(g["rho"]), float(g["dt"]), 1e-10, 500, p=p, DP=DP)
    torch.cuda.synchronize()
    assert info.status == 0 and info.max_res <= 1e-10
    s = np.abs(g["DP"]).max()
    assert np.abs(DP.cpu().numpy() - g["DP"]).max() <= 2e-8 * s
    assert np.abs(p.cpu().numpy() - g["p_out"]).max() <= 2e-8 * s
    for t, k in zip(tgt, ("u_out", "v_out", "w_out")):
        assert np.abs(t.cpu().numpy() - g[k]).max() <= 1e-9 * np.abs(g[k]).max(), k
    # the corrected target is discretely divergence free to the solver tolerance
    div = ops.div_vel(*tgt, g["spacing"]).abs().max().item()
    div0 = ops.div_vel(*(cu(g[k]) for k in ("uT", "vT", "wT")), g["spacing"]).abs().max().item()
    assert div <= 1e-8 * div0
