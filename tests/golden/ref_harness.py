"""Harness that runs the unmodified reference PyFlow (pure Python/PyTorch, CPU)
in this container, to generate golden fixtures for the oracle and the CUDA path.

It is used only by ``make_golden.py``; nothing on the GPU side imports it.  The
reference tree is copied to a temporary directory (the reference writes
``monitor/`` and restart files relative to its working directory) and imported
with three shims:

* a single-rank fake ``mpi4py`` and a stub ``matplotlib`` (``refshim/``);
* ``geometry.Geometry_Base`` -> ``geometry.uniform`` (src/core/PyFlow.py:103
  calls a class that src/geometry/geometry.py never defines);
* serial NGA restart readers/writers in place of the MPI-IO ones
  (src/data/dataReader.py:215-390), using the same file format as the serial
  reader at src/data/dataReader.py:119-208.
"""
import os
import shutil
import struct
import sys
import tempfile
import types

import numpy as np

# root of the reference checkout (the directory holding its src/); required
REF_ROOT = os.environ.get("PF_REFERENCE_ROOT")
HERE = os.path.dirname(os.path.abspath(__file__))

_loaded = {}


def load_reference():
    """Copy the reference ``src/`` to a temp dir, install the shims and import
    its modules.  Returns a namespace of the reference modules."""
    if "ns" in _loaded:
        return _loaded["ns"]
    if not REF_ROOT or not os.path.isdir(os.path.join(REF_ROOT, "src")):
        raise RuntimeError("set PF_REFERENCE_ROOT to the reference checkout (the directory "
                           "that holds its src/)")
    import torch  # noqa: F401  (the reference imports torch itself)

    tmp = tempfile.mkdtemp(prefix="pyflow_ref_")
    src = os.path.join(tmp, "src")
    shutil.copytree(os.path.join(REF_ROOT, "src"), src)
    sys.path.insert(0, os.path.join(HERE, "refshim"))
    for sub in ("core", "data", "library", "geometry", "metric", "solver",
                "sfsmodel", "boundary"):
        sys.path.insert(0, os.path.join(src, sub))
    os.chdir(os.path.join(src, "core"))

    import geometry
    import dataReader
    import parallel
    import metric_staggered
    import state
    import velocity
    import pressure
    import advancer
    import domain
    import sfsmodel_smagorinsky
    import sfsmodel_gradient
    import sfsmodel_ML
    import adjoint
    import PyFlow

    geometry.Geometry_Base = (
        lambda IC, x, y, z, d: geometry.uniform(x, y, z, d))

    def read_restart_serial(fName, data_all_CPU, ivar_read_start=None,
                            nvar_read=None):
        names, time, data = read_restart(fName)
        for ivar in range(data_all_CPU.nvar_read):
            data_all_CPU.append(ivar, np.ascontiguousarray(data[..., ivar]))

    def write_restart_serial(fName, data_all_CPU):
        pass

    dataReader.readNGArestart_parallel = read_restart_serial
    dataReader.writeNGArestart_parallel = write_restart_serial
    dataReader.writeNGArestart = lambda *a, **k: None
    # domain.py and PyFlow.py import dataReader as dr at module level
    PyFlow.dr = dataReader
    domain.dr = dataReader

    ns = types.SimpleNamespace(
        geometry=geometry, dataReader=dataReader, parallel=parallel,
        metric_staggered=metric_staggered, state=state, velocity=velocity,
        pressure=pressure, advancer=advancer, domain=domain,
        sfsmodel_smagorinsky=sfsmodel_smagorinsky,
        sfsmodel_gradient=sfsmodel_gradient, sfsmodel_ML=sfsmodel_ML, adjoint=adjoint, PyFlow=PyFlow,
        tmp=tmp)
    _loaded["ns"] = ns
    return ns


# ---------------------------------------------------------------------------
# NGA file writers (format of src/data/dataReader.py:60-112 and :119-208)
# ---------------------------------------------------------------------------
def write_config(fname, xg, yg, zg, per=(1, 1, 1)):
    with open(fname, "wb") as f:
        f.write(b"pyflow_b200".ljust(64))
        f.write(struct.pack("<7i", 0, per[0], per[1], per[2],
                            len(xg) - 1, len(yg) - 1, len(zg) - 1))
        for g in (xg, yg, zg):
            f.write(np.asarray(g, dtype="<f8").tobytes())


def write_restart(fname, fields, names=("U", "V", "W", "P"), dt=0.0, time=0.0):
    nx, ny, nz = fields[0].shape
    with open(fname, "wb") as f:
        f.write(struct.pack("<4i", nx, ny, nz, len(fields)))
        f.write(struct.pack("<2d", dt, time))
        for n in names:
            f.write(n.ljust(8).encode())
        for a in fields:
            f.write(np.asarray(a, dtype="<f8").reshape(-1, order="F").tobytes())


def read_restart(fname):
    with open(fname, "rb") as f:
        nx, ny, nz, nvar = struct.unpack("<4i", f.read(16))
        dt, time = struct.unpack("<2d", f.read(16))
        names = [f.read(8).decode().strip() for _ in range(nvar)]
        data = np.empty((nx, ny, nz, nvar))
        for v in range(nvar):
            data[..., v] = np.frombuffer(
                f.read(8 * nx * ny * nz), dtype="<f8").reshape(
                    (nx, ny, nz), order="F")
    return names, time, data


# ---------------------------------------------------------------------------
# Per-operator objects on a single rank
# ---------------------------------------------------------------------------
class _IC:
    pass


def make_setup(nx, ny, nz, lx, ly, lz):
    """Build the reference's comms/decomp/geometry/metric for a periodic box."""
    import torch
    ns = load_reference()
    IC = _IC()
    IC.dtypeTorch = torch.float64
    IC.dtypeNumpy = np.float64
    IC.nproc_x = IC.nproc_y = IC.nproc_z = 1
    cfg = _IC()
    cfg.Nx, cfg.Ny, cfg.Nz = nx, ny, nz
    cfg.isper = [1, 1, 1]
    comms = ns.parallel.comms(IC)
    decomp = ns.parallel.decomp(IC, cfg)
    xg = np.linspace(0.0, lx, nx + 1)
    yg = np.linspace(0.0, ly, ny + 1)
    zg = np.linspace(0.0, lz, nz + 1)
    geo = ns.geometry.uniform(xg, yg, zg, decomp)
    metric = ns.metric_staggered.metric_uniform(geo)
    return types.SimpleNamespace(ns=ns, IC=IC, comms=comms, decomp=decomp,
                                 geo=geo, metric=metric)


def padded(decomp, interior):
    """An [n+4]^3 torch tensor holding ``interior`` with periodic ghosts."""
    import torch
    t = torch.zeros(decomp.nxo_, decomp.nyo_, decomp.nzo_, dtype=torch.float64)
    t[2:-2, 2:-2, 2:-2] = torch.from_numpy(interior)
    decomp.communicate_border(t)
    return t
