"""The reference's 'source' ML closure (pyflow_b200.sfsmodel_ML) against the
reference itself (tests/golden/ml_16.npz: rhs_NavierStokes.evaluate with a
seeded network whose weights the fixture stores).

The reference wraps its shifts around ghost-padded arrays, which changes its
closure on the three cells nearest each periodic boundary; the comparison is
on the cells at least three cells away (indices 3 .. n-4)."""
import numpy as np
import pytest
import torch

import oracle as O


def _model(g):
    import pyflow_b200.sfsmodel_ML as M
    net = M.GatedClosureNet()
    sd = {k[2:]: torch.from_numpy(np.asarray(g[k])) for k in g if k.startswith("w_")}
    net.load_state_dict(sd)
    return net


class _Geo:
    type = "uniform"

    def __init__(self, dx):
        self.dx = dx


class _Decomp:
    def __init__(self, device):
        self.device = device


def _source(g, device):
    import pyflow_b200.sfsmodel_ML as M

    class IC:
        simDt = 0.01

    ml = M.residual_stress(IC(), _Decomp(device), _Geo(float(g["spacing"][0])),
                           model=_model(g))
    u, v, w = (torch.tensor(g[k], device=device) for k in ("u", "v", "w"))
    ml.update(u, v, w)
    return [t.cpu().numpy() for t in ml.face_sources()]


def test_ml_source_matches_reference_cpu(golden):
    """Restatement check on the CPU: oracle RHS minus our face sources."""
    g = golden("ml_16.npz")
    plain = O.rhs_ns(g["spacing"], g["u"], g["v"], g["w"], float(g["mu"]), float(g["rho"]))
    src = _source(g, "cpu")
    n = int(g["shape"][0])
    sl = (slice(3, n - 3),) * 3
    for c in range(3):
        got = (plain[c] - src[c])[sl]
        ref = g["rhs_ml"][c][sl]
        assert np.abs(got - ref).max() <= 1e-5 * np.abs(ref).max()


@pytest.mark.gpu
def test_ml_source_rhs_gpu(golden):
    """The drop-in RHS object with the ML closure on the GPU."""
    import pyflow_b200.sfsmodel_ML as M
    import pyflow_b200.velocity as V
    g = golden("ml_16.npz")
    n = int(g["shape"][0])

    class IC:
        simDt = 0.01

    class Dec:
        nx_ = ny_ = nz_ = n
        device = torch.device("cuda")

    class Met:
        spacing = tuple(float(x) for x in g["spacing"])

    class St:
        def __init__(self, a):
            self.a = torch.tensor(a, device="cuda")

        def interior(self):
            return self.a

    ml = M.residual_stress(IC(), Dec(), _Geo(float(g["spacing"][0])), model=_model(g))
    r = V.rhs_NavierStokes(Dec(), Met(), float(g["rho"]), float(g["mu"]), ml)
    r.evaluate(St(g["u"]), St(g["v"]), St(g["w"]))
    sl = (slice(3, n - 3),) * 3
    for c, t in enumerate((r.rhs_u, r.rhs_v, r.rhs_w)):
        ref = g["rhs_ml"][c][sl]
        assert np.abs(t.cpu().numpy()[sl] - ref).max() <= 1e-5 * np.abs(ref).max()
