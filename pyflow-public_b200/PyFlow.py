"""PyFlow.run(inputConfig) -- the reference's driver contract
(src/core/PyFlow.py:69-666) on the B200 path.

Reads the same duck-typed ``inputConfig`` attributes, sets up the periodic
box from an NGA config + restart file (or a seeded spectral field with
``configName='spectral'``), advances ``numIt`` steps with Domain.forwardStep,
prints the reference's per-step table and writes ``monitor/velocity_<case>.txt``
and NGA restart files (``fNameOut_<time>``, every ``numItDataOut`` steps and at
the end).  Per-step statistics come from one fused reduction kernel and one
40-byte device-to-host read.

Adjoint training/verification (src/core/PyFlow.py:312-607) runs through
pyflow_b200.adjoint when ``adjointTraining`` is set.
"""
import os
import time

import numpy as np
import torch

from . import dataReader as dr
from . import domain as dom
from . import geometry as geo
from . import metric_staggered
from . import ops
from . import parallel


class DeviceIC:
    """The initial state as device fields, indexed like the reference's
    data_IC[..., v]."""

    def __init__(self, fields):
        self.fields = fields
        self.shape = tuple(fields[0].shape) + (len(fields),)

    def __getitem__(self, key):
        if isinstance(key, tuple) and len(key) == 2 and key[0] is Ellipsis:
            return self.fields[key[1]]
        raise IndexError("DeviceIC supports data_IC[..., v] only")


def _initial_data(inputConfig, config, decomp):
    """names, startTime, data_IC[nx,ny,nz,4] (src/data/initial_conditions.py:39-77)."""
    name = getattr(inputConfig, "configName", "restart")
    if name == "restart":
        # straight into device memory (src/data/initial_conditions.py:57-77
        # reads the restart into host arrays first)
        (nx, ny, nz, nv), _, _ = dr.readNGArestart_dims(inputConfig.dataFileStr)
        if (nx, ny, nz) != (config.Nx, config.Ny, config.Nz):
            raise ValueError("restart file and config grid sizes differ")
        names, t0, fields = dr.readNGArestart_device(inputConfig.dataFileStr, decomp.device,
                                                     nvar=4)
        while len(fields) < 4:
            fields.append(torch.zeros_like(fields[0]))
        return ["U", "V", "W", "P"], t0, DeviceIC(fields)
    if name == "spectral":
        from . import initial
        L = (config.xGrid[-1] - config.xGrid[0], config.yGrid[-1] - config.yGrid[0],
             config.zGrid[-1] - config.zGrid[0])
        u, v, w = initial.spectral_velocity(
            (config.Nx, config.Ny, config.Nz), lengths=L,
            k0=getattr(inputConfig, "k0", 4.0), urms=getattr(inputConfig, "urms", 1.0),
            seed=getattr(inputConfig, "seed", 0))
        out = np.stack([u, v, w, np.zeros_like(u)], axis=-1)
        return ["U", "V", "W", "P"], getattr(inputConfig, "startTime", 0.0), out
    raise ValueError("configName %r not supported (the reference's analytic "
                     "initial conditions are broken; use 'restart' or 'spectral')" % name)


def _stats(D, geometry):
    st = ops.stats(D.state_u_P.interior(), D.state_v_P.interior(),
                   D.state_w_P.interior(), geometry.spacing).cpu().numpy()
    return st  # max|u|, max|v|, max|w|, TKE, max|div u|


def run(inputConfig):
    comms = parallel.comms(inputConfig)
    config = geo.config(inputConfig)
    decomp = parallel.decomp(inputConfig, config)
    numPoints = decomp.nx * decomp.ny * decomp.nz
    names, startTime, data_IC = _initial_data(inputConfig, config, decomp)
    geometry = geo.Geometry_Base(inputConfig, config.xGrid, config.yGrid,
                                 config.zGrid, decomp)
    metric = metric_staggered.metric_uniform(geometry)
    D = dom.Domain(inputConfig, comms, decomp, data_IC, geometry, metric, names,
                   startTime)
    del data_IC

    if getattr(inputConfig, "adjointTraining", False):
        from . import adjoint
        return adjoint.run_training(inputConfig, comms, decomp, geometry, metric, D,
                                    startTime)

    simDt = inputConfig.simDt
    simTime = startTime
    stopTime = startTime + inputConfig.numIt * simDt
    rank0 = decomp.rank == 0
    fNameOut = getattr(inputConfig, "fNameOut", None)
    numItDataOut = getattr(inputConfig, "numItDataOut", 0) or 0

    def write_restart(t):
        if fNameOut and rank0:
            D.data_all_CPU.time, D.data_all_CPU.dt = t, simDt
            dr.writeNGArestart_device(fNameOut + "_" + "{:12.7E}".format(t),
                                      [s.interior() for s in D.state_data_all],
                                      D.data_all_CPU.names, simDt, t)

    write_restart(simTime)
    if rank0:
        print("\n  {:10s}   {:9s}   {:9s}   {:9s}   {:9s}   {:9s}   {:9s}   {:9s}   {:9s}".format(
            "Step", "Time", "max CFL", "max U", "max V", "max W", "TKE", "divergence",
            "max res_P"))
    st = _stats(D, geometry)
    TKE = st[3]
    initEnergy = TKE
    maxU, maxV, maxW, maxDivg = st[0], st[1], st[2], st[4]
    maxCFL = max((maxU / geometry.dx, maxV / geometry.dy, maxW / geometry.dz)) * simDt
    lineStr = "  {:10d}   {:8.3E}   {:8.3E}   {:8.3E}   {:8.3E}   {:8.3E}   {:8.3E}   {:8.3E}"
    monitorFile = None
    if rank0:
        print(lineStr.format(0, simTime, maxCFL, maxU, maxV, maxW, TKE, maxDivg))
        os.makedirs("monitor", exist_ok=True)
        caseName = getattr(inputConfig, "caseName", "PyFlow")
        monitorFile = open("monitor/velocity_" + caseName + ".txt", "w")
        monitorFile.write("  {:10s}   {:9s}   {:9s}   {:9s}   {:9s}   {:9s}   {:9s}   {:9s}   {:9s} \n".format(
            "Step", "Time", "max CFL", "max U", "max V", "max W", "TKE", "divergence", "max res_P"))
        monitorFile.write((lineStr + "\n").format(0, simTime, maxCFL, maxU, maxV, maxW, TKE, maxDivg))

    time1 = time.time()
    itCount = 0
    viscNu = inputConfig.mu / inputConfig.rho
    history = []
    while simTime < stopTime and itCount < inputConfig.numIt:
        D.forwardStep(simDt)
        itCount += 1
        simTime += simDt
        st = _stats(D, geometry)
        maxU, maxV, maxW, TKE, maxDivg = st
        maxCFL = max((maxU / geometry.dx, maxV / geometry.dy, maxW / geometry.dz)) * simDt
        maxVNN = max((viscNu / geometry.dx ** 2, viscNu / geometry.dy ** 2,
                      viscNu / geometry.dz ** 2)) * simDt
        maxCFL = max((maxCFL, maxVNN))
        history.append((itCount, simTime, maxCFL, maxU, maxV, maxW, TKE, maxDivg, D.max_resP))
        if rank0:
            line = ("  {:10d}   {:8.3E}   {:8.3E}   {:8.3E}   {:8.3E}   {:8.3E}   {:8.3E}   {:8.3E}   {:8.3E}"
                    .format(itCount, simTime, maxCFL, maxU, maxV, maxW, TKE, maxDivg, D.max_resP))
            print(line)
            monitorFile.write(line + "\n")
        if numItDataOut and itCount % numItDataOut == 0:
            write_restart(simTime)

    write_restart(simTime)
    time_elapsed = time.time() - time1
    finalEnergy = float(_stats(D, geometry)[3])
    test = float(torch.mean(D.state_u_P.interior()))
    if rank0:
        print("\nit={}, test={:10.5E}, elapsed={}".format(itCount, test, time_elapsed))
        print("Energy initial={:10.5E}, final={:10.5E}, ratio={:10.5E}".format(
            initEnergy, finalEnergy, finalEnergy / initEnergy if initEnergy else float("nan")))
        monitorFile.close()
    run.last_domain = D
    run.last_history = history
    return None
