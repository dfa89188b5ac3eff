"""NGA config / restart files (format of src/data/dataReader.py:60-208).

Serial numpy readers and writers: the restart format is a header
``<4i nx,ny,nz,nvar><2d dt,time><8-char names>`` followed by each variable in
Fortran order (float64).  Used by PyFlow.run for initial conditions and
checkpoint/resume; device fields are copied in and out whole.
"""
import struct

import numpy as np


def readNGAconfig(fName):
    """(xGrid, yGrid, zGrid, xper, yper, zper) of an NGA config file
    (src/data/dataReader.py:60-112)."""
    with open(fName, "rb") as f:
        f.read(64)
        icyl, xper, yper, zper, nx, ny, nz = struct.unpack("<7i", f.read(28))
        xg = np.frombuffer(f.read(8 * (nx + 1)), dtype="<f8").copy()
        yg = np.frombuffer(f.read(8 * (ny + 1)), dtype="<f8").copy()
        zg = np.frombuffer(f.read(8 * (nz + 1)), dtype="<f8").copy()
    return xg, yg, zg, xper, yper, zper


def writeNGAconfig(fName, xGrid, yGrid, zGrid, per=(1, 1, 1), name="pyflow"):
    with open(fName, "wb") as f:
        f.write(name.encode()[:64].ljust(64))
        f.write(struct.pack("<7i", 0, per[0], per[1], per[2], len(xGrid) - 1,
                            len(yGrid) - 1, len(zGrid) - 1))
        for g in (xGrid, yGrid, zGrid):
            f.write(np.asarray(g, dtype="<f8").tobytes())


def readNGArestart(fName, headerOnly=True, printOut=False):
    """(names, time) or (names, time, data[nx,ny,nz,nvar]) of a restart file
    (src/data/dataReader.py:119-171)."""
    with open(fName, "rb") as f:
        nx, ny, nz, nvar = struct.unpack("<4i", f.read(16))
        dt, time = struct.unpack("<2d", f.read(16))
        names = [f.read(8).decode().strip() for _ in range(nvar)]
        if headerOnly:
            return names, time
        data = np.empty((nx, ny, nz, nvar))
        for v in range(nvar):
            data[..., v] = np.frombuffer(f.read(8 * nx * ny * nz), dtype="<f8").reshape(
                (nx, ny, nz), order="F")
    return names, time, data


def readNGArestart_dims(fName):
    with open(fName, "rb") as f:
        nx, ny, nz, nvar = struct.unpack("<4i", f.read(16))
        dt, time = struct.unpack("<2d", f.read(16))
    return (nx, ny, nz, nvar), dt, time


def writeNGArestart(fName, fields, names, dt, time):
    """Write host arrays ``fields`` (each [nx,ny,nz]) as a restart file
    (src/data/dataReader.py:179-208)."""
    nx, ny, nz = fields[0].shape
    with open(fName, "wb") as f:
        f.write(struct.pack("<4i", nx, ny, nz, len(fields)))
        f.write(struct.pack("<2d", dt, time))
        for n in names:
            f.write(n.ljust(8)[:8].encode())
        for a in fields:
            f.write(np.asarray(a, dtype="<f8").reshape(-1, order="F").tobytes())
