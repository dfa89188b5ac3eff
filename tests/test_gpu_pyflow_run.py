"""The drop-in driver contract: a reference-style input configuration runs
unchanged through pyflow_b200.PyFlow.run and reproduces the reference's own
PyFlow.run (tests/golden/run_32.npz, 5 RK4 + BiCGStab steps at 32^3), through
the same NGA config/restart files and monitor output."""
import os

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


class inputConfigClass:
    """Attribute set of the reference's example driver
    (examples/dnsbox_128/run_PyFlow_example_dnsbox128.py:43-98)."""

    def __init__(self, wd, g, solver="bicgstab", precision=None):
        self.configName = "restart"
        self.configFileStr = os.path.join(wd, "config")
        self.dataFileStr = os.path.join(wd, "data")
        self.dataFileType = "restart"
        self.fNameOut = os.path.join(wd, "out")
        self.numItDataOut = 1000
        self.nproc_x = self.nproc_y = self.nproc_z = 1
        self.mu = float(g["nu"])
        self.rho = float(g["rho"])
        self.simDt = float(g["dt"])
        self.numIt = int(g["steps"])
        self.startTime = 0.0
        self.SFSmodel = "none"
        self.advancerName = "RK4"
        self.equationMode = "NS"
        self.pSolverMode = solver
        self.min_pressure_residual = 1e-10
        self.max_pressure_iterations = 1000
        self.genericOrder = 2
        self.dtypeTorch = torch.float64
        self.dtypeNumpy = np.float64
        self.plotState = False
        self.numItPlotOut = 20
        if precision:
            self.precisionMode = precision


def _write_inputs(wd, g):
    import pyflow_b200.dataReader as dr
    n = int(g["shape"][0])
    grid = np.linspace(0.0, 2 * np.pi, n + 1)
    dr.writeNGAconfig(os.path.join(wd, "config"), grid, grid, grid)
    dr.writeNGArestart(os.path.join(wd, "data"),
                       [g["u0"], g["v0"], g["w0"], np.zeros_like(g["u0"])],
                       ["U", "V", "W", "P"], float(g["dt"]), 0.0)


@pytest.mark.parametrize("precision,tol", [(None, 1e-9), ("mixed", 1e-6), ("mixed_mg", 1e-6)])
def test_pyflow_run_matches_reference(golden, tmp_path, monkeypatch, precision, tol):
    import pyflow_b200.PyFlow as PyFlow
    import pyflow_b200.dataReader as dr
    g = golden("run_32.npz")
    monkeypatch.chdir(tmp_path)
    _write_inputs(str(tmp_path), g)
    assert PyFlow.run(inputConfigClass(str(tmp_path), g, precision=precision)) is None
    outs = sorted(f for f in os.listdir(tmp_path) if f.startswith("out_"))
    assert len(outs) == 2  # initial and final restart files
    names, t, data = dr.readNGArestart(os.path.join(tmp_path, outs[-1]), headerOnly=False)
    assert names == ["U", "V", "W", "P"]
    assert abs(t - int(g["steps"]) * float(g["dt"])) < 1e-12
    for c, key in enumerate(("u", "v", "w")):
        ref = g[key]
        assert np.abs(data[..., c] - ref).max() <= tol * np.abs(ref).max()
    hist = PyFlow.run.last_history
    assert len(hist) == int(g["steps"])
    for s, row in enumerate(hist):
        np.testing.assert_allclose(row[6], g["stats"][s][3], rtol=max(tol, 1e-11))
    mon = open(os.path.join(tmp_path, "monitor", "velocity_PyFlow.txt")).read().splitlines()
    assert len(mon) == 2 + int(g["steps"])


def test_pyflow_run_jacobi(golden, tmp_path, monkeypatch):
    """The Jacobi path (fixed sweeps) runs through the driver and reduces the
    divergence like the reference's solver_jacobi."""
    import pyflow_b200.PyFlow as PyFlow
    g = golden("run_32.npz")
    monkeypatch.chdir(tmp_path)
    _write_inputs(str(tmp_path), g)
    cfg = inputConfigClass(str(tmp_path), g, solver="Jacobi")
    cfg.max_pressure_iterations = 50
    cfg.numIt = 2
    PyFlow.run(cfg)
    hist = PyFlow.run.last_history
    assert len(hist) == 2 and all(np.isfinite(h[7]) for h in hist)


def test_pyflow_run_with_reference_ml_model(golden, tmp_path, monkeypatch):
    """SFSmodel='ML' with loadModel: a checkpoint in the reference's format
    (epoch, LR, model_state_dict) drives the 'source' closure at every RK
    stage through the driver; the run stays finite and divergence free and
    differs from the run without the closure."""
    import torch
    import pyflow_b200.PyFlow as PyFlow
    gm = golden("ml_16.npz")
    sd = {k[2:]: torch.from_numpy(np.asarray(gm[k])) for k in gm if k.startswith("w_")}
    ck = os.path.join(str(tmp_path), "model.dict")
    torch.save({"epoch": 3, "LR": 0.01, "model_state_dict": sd}, ck)
    g = golden("run_32.npz")
    monkeypatch.chdir(tmp_path)
    _write_inputs(str(tmp_path), g)
    hist = {}
    for name in ("none", "ML"):
        cfg = inputConfigClass(str(tmp_path), g)
        cfg.numIt = 2
        cfg.SFSmodel = name
        cfg.loadModel = True
        cfg.modelDictName = ck
        PyFlow.run(cfg)
        hist[name] = PyFlow.run.last_history
    assert all(np.isfinite(r).all() for r in hist["ML"])
    assert hist["ML"][-1][7] < 1e-8          # max |div u| after the projection
    assert abs(hist["ML"][-1][6] - hist["none"][-1][6]) > 0.0
