"""The reference's 'source' ML closure (pyflow_b200.sfsmodel_ML) against the
reference itself (tests/golden/ml_16.npz: rhs_NavierStokes.evaluate with a
seeded network whose weights the fixture stores).

The reference wraps its shifts around ghost-padded arrays, which changes its
closure on the three cells nearest each periodic boundary; the comparison of
the periodic closure is on the cells at least three cells away (indices
3 .. n-4).  The remaining cells are pinned by feeding the same closure
pipeline the reference's own inputs (the fixture's ``ci``: its ghost-padded
cell-centre interpolants, whose last ghost layer its interpolation never
writes): on those, every cell of the RHS matches bit for bit, and ``ci``
equals the periodic interpolant everywhere but that layer."""
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


def test_ml_source_all_cells_on_reference_inputs(golden):
    """Features, 13-point network input, gated network, closure terms and
    face sources (the same functions the periodic closure uses), evaluated on
    the reference's ghost-padded closure inputs with its wrap-around shifts:
    the RHS matches the reference's on every cell, bit for bit."""
    import pyflow_b200.sfsmodel_ML as M
    g = golden("ml_16.npz")
    dx, h = float(g["spacing"][0]), 2
    C = [torch.tensor(g["ci"][c]).to(torch.float32) for c in range(3)]
    first, second = [], []
    for a in C:
        d1, d2 = M._derivatives(a, dx)
        first += d1
        second += d2
    F = torch.stack(C + first + second, dim=3)
    norm = torch.tensor(M.NORM, dtype=torch.float32)
    with torch.no_grad():
        p = _model(g)(M.network_input(F, norm))
    G = [t.double() for t in M.closure_terms(p, dx)]
    plain = O.rhs_ns(g["spacing"], g["u"], g["v"], g["w"], float(g["mu"]), float(g["rho"]))
    for ax in range(3):
        # interp_sc_x/y/z (src/metric/metric_staggered.py:112-124) on the
        # padded array, then the interior
        lo = [slice(None)] * 3
        hi = [slice(None)] * 3
        lo[ax], hi[ax] = slice(0, -1), slice(1, None)
        face = torch.zeros_like(G[ax])
        face[tuple(hi)] = 0.5 * (G[ax][tuple(hi)] + G[ax][tuple(lo)])
        got = plain[ax] - face.numpy()[h:-h, h:-h, h:-h]
        assert np.array_equal(got, g["rhs_ml"][ax])


def test_ml_source_reference_inputs_differ_only_in_stale_layer(golden):
    """The reference's closure inputs are the periodic cell-centre
    interpolants of the padded velocity except on the last ghost layer along
    each component's own axis, which its interpolation never writes
    (src/metric/metric_staggered.py:149-152): that layer is the whole
    difference between the reference's boundary cells and the periodic
    closure."""
    g = golden("ml_16.npz")
    for ax, k in enumerate(("u", "v", "w")):
        pad = np.pad(g[k], 2, mode="wrap")
        want = 0.5 * (np.roll(pad, -1, ax) + pad)
        ci = g["ci"][ax]
        keep = [slice(None)] * 3
        keep[ax] = slice(0, -1)
        assert np.array_equal(ci[tuple(keep)], want[tuple(keep)])
        last = [slice(None)] * 3
        last[ax] = -1
        assert not np.array_equal(ci[tuple(last)], want[tuple(last)])


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
