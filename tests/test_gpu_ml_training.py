"""Training the reference's 'source' ML closure through the hand-written
adjoint: the gradients of a multi-step objective with respect to the initial
velocity and to the network weights against central differences (closure
evaluated in FP64 so the objective is smooth), and the adjointTraining /
adjointVerification modes of PyFlow.run end to end."""
import math
import os

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


class _Geo:
    type = "uniform"

    def __init__(self, dx):
        self.dx = dx


class _Dec:
    device = torch.device("cuda")


def _model(seed=3, scale=0.2):
    import pyflow_b200.sfsmodel_ML as M
    torch.manual_seed(seed)
    net = M.GatedClosureNet()
    with torch.no_grad():
        net.fc4.weight.mul_(scale)
    return net


def _closure(n, net, dtype="float64"):
    import pyflow_b200.sfsmodel_ML as M

    class IC:
        simDt = 0.01
        mlDtype = dtype

    return M.residual_stress(IC(), _Dec(), _Geo(2 * math.pi / n), model=net)


def test_source_step_gradients_match_finite_differences():
    import pyflow_b200.adjoint as A
    import pyflow_b200.initial as ic
    n = 16
    sp = (2 * math.pi / n,) * 3
    ml = _closure(n, _model())
    src = A.source_fn(ml)
    f0 = [torch.tensor(a, device="cuda") for a in ic.spectral_velocity((n,) * 3, seed=8)]
    rng = np.random.default_rng(2)
    wts = [torch.tensor(rng.standard_normal((n,) * 3), device="cuda") for _ in range(3)]

    def objective(u0, steps=2):
        cur = tuple(u0)
        for _ in range(steps):
            cur = A.forward_step(*cur, sp, 0.02, 1.0, 0.01, tol=1e-13, source=src)
        return sum((c * w).sum() for c, w in zip(cur, wts))

    u0 = [t.clone().requires_grad_(True) for t in f0]
    ml.model.zero_grad()
    L = objective(u0)
    L.backward()
    # velocity direction
    d = [torch.tensor(rng.standard_normal((n,) * 3), device="cuda") for _ in range(3)]
    g = sum(float((a.grad * b).sum()) for a, b in zip(u0, d))
    eps = 1e-6
    with torch.no_grad():
        lp = float(objective([a + eps * b for a, b in zip(f0, d)]))
        lm = float(objective([a - eps * b for a, b in zip(f0, d)]))
    fd = (lp - lm) / (2 * eps)
    assert abs(fd - g) <= 1e-5 * abs(g), (fd, g)
    # weight direction (output layer)
    W = ml.model.fc4.weight
    gw = W.grad.detach().clone()
    dW = torch.tensor(rng.standard_normal(tuple(W.shape)), dtype=W.dtype, device="cuda")
    gdir = float((gw * dW).sum())
    base = W.detach().clone()
    eps = 1e-5
    with torch.no_grad():
        W.copy_(base + eps * dW)
        lp = float(objective(f0))
        W.copy_(base - eps * dW)
        lm = float(objective(f0))
        W.copy_(base)
    fd = (lp - lm) / (2 * eps)
    assert abs(gdir) > 0
    assert abs(fd - gdir) <= 1e-5 * abs(gdir), (fd, gdir)


def _inputs(wd, n, seed=0):
    import pyflow_b200.dataReader as dr
    import pyflow_b200.initial as ic
    grid = np.linspace(0.0, 2 * np.pi, n + 1)
    dr.writeNGAconfig(os.path.join(wd, "config"), grid, grid, grid)
    u, v, w = ic.spectral_velocity((n,) * 3, seed=seed)
    dr.writeNGArestart(os.path.join(wd, "data"), [u, v, w, np.zeros_like(u)],
                       ["U", "V", "W", "P"], 0.01, 0.0)
    return u, v, w


class _Cfg:
    def __init__(self, wd, model_path):
        self.configName = "restart"
        self.configFileStr = os.path.join(wd, "config")
        self.dataFileStr = os.path.join(wd, "data")
        self.dataFileType = "restart"
        self.fNameOut = os.path.join(wd, "out")
        self.numItDataOut = 1000
        self.nproc_x = self.nproc_y = self.nproc_z = 1
        self.mu, self.rho, self.simDt = 0.02, 1.0, 0.01
        self.startTime = 0.0
        self.SFSmodel = "ML"
        self.advancerName = "RK4"
        self.equationMode = "NS"
        self.pSolverMode = "bicgstab"
        self.min_pressure_residual = 1e-13
        self.max_pressure_iterations = 5000
        self.genericOrder = 2
        self.dtypeTorch = torch.float64
        self.dtypeNumpy = np.float64
        self.plotState = False
        self.numItPlotOut = 20
        self.adjointTraining = True
        self.loadModel = True
        self.modelDictName = model_path
        self.mlDtype = "float64"


def test_pyflow_adjoint_verification_matches_finite_difference(tmp_path, monkeypatch):
    import pyflow_b200.PyFlow as PyFlow
    n = 16
    wd = str(tmp_path)
    monkeypatch.chdir(tmp_path)
    _inputs(wd, n)
    ck = os.path.join(wd, "model.dict")
    torch.save({"epoch": 0, "LR": 0.01, "model_state_dict": _model().state_dict()}, ck)

    def run(pert):
        cfg = _Cfg(wd, ck)
        cfg.numIt, cfg.numCheckpointIt = 2, 2
        cfg.adjointVerification = True
        cfg.perturbation = pert
        return PyFlow.run(cfg)

    obj, grad = run(0.0)
    eps = 1e-4
    fd = (run(eps)[0] - run(-eps)[0]) / (2 * eps)
    assert abs(grad) > 0
    assert abs(fd - grad) <= 1e-4 * abs(grad), (fd, grad)


def test_pyflow_adjoint_training_updates_model(tmp_path, monkeypatch):
    import pyflow_b200.PyFlow as PyFlow
    import pyflow_b200.dataReader as dr
    import pyflow_b200.initial as ic
    n = 16
    wd = str(tmp_path)
    monkeypatch.chdir(tmp_path)
    _inputs(wd, n)
    # targets after 2 and 4 steps: another seeded field
    for it in (2, 4):
        u, v, w = ic.spectral_velocity((n,) * 3, seed=40 + it)
        dr.writeNGArestart(os.path.join(wd, "target_%d" % it), [u, v, w, np.zeros_like(u)],
                           ["U", "V", "W", "P"], 0.01, 0.01 * it)
    net = _model()
    ck = os.path.join(wd, "model.dict")
    torch.save({"epoch": 0, "LR": 0.01, "model_state_dict": net.state_dict()}, ck)
    cfg = _Cfg(wd, ck)
    cfg.mlDtype = "float32"
    cfg.numIt, cfg.numCheckpointIt = 4, 2
    cfg.startFileIt = 0
    cfg.getTargetFileName = lambda it: os.path.join(wd, "target_%d" % it)
    cfg.targetDataVelCorr = True
    cfg.modelDictSave = os.path.join(wd, "model_out.dict")
    cfg.numSumDistr = 1
    assert PyFlow.run(cfg) is None
    out = torch.load(cfg.modelDictSave)
    assert out["epoch"] == 2
    w0 = net.state_dict()["fc1.weight"].cpu()
    w1 = out["model_state_dict"]["fc1.weight"].cpu()
    assert not torch.equal(w0, w1)
    import pyflow_b200.adjoint as A
    hist = A.run_training.last_history
    assert len(hist) == 4 and all(np.isfinite(h).all() for h in hist)
    assert hist[1][-1] > 0 and hist[3][-1] > 0   # window objectives
