"""Grid configuration with the reference's interface (src/geometry/geometry.py).

``config(IC)`` reads the grid from an NGA config file for restarts
(src/geometry/geometry.py:40-70); ``uniform(x, y, z, decomp)`` computes the
uniform spacings (:76-116).  ``Geometry_Base`` is what src/core/PyFlow.py:103
calls (a name the reference never defines); here it is ``uniform``.
"""
import numpy as np

from . import dataReader as dr


class config:
    def __init__(self, IC):
        name = getattr(IC, "configName", "restart")
        if name == "restart":
            if getattr(IC, "dataFileType", "restart") != "restart":
                raise ValueError("only NGA restart input is supported "
                                 "(the reference's volume path raises too)")
            (self.xGrid, self.yGrid, self.zGrid,
             xper, yper, zper) = dr.readNGAconfig(IC.configFileStr)
            self.Nx, self.Ny, self.Nz = (len(self.xGrid) - 1, len(self.yGrid) - 1,
                                         len(self.zGrid) - 1)
            self.isper = [xper, yper, zper]
        else:
            # generated fields (pyflow_b200.initial) on a periodic box
            self.Nx, self.Ny, self.Nz = IC.Nx, IC.Ny, IC.Nz
            L = getattr(IC, "Lx", 2 * np.pi), getattr(IC, "Ly", 2 * np.pi), getattr(IC, "Lz", 2 * np.pi)
            self.xGrid = np.linspace(0.0, L[0], self.Nx + 1)
            self.yGrid = np.linspace(0.0, L[1], self.Ny + 1)
            self.zGrid = np.linspace(0.0, L[2], self.Nz + 1)
            self.isper = [1, 1, 1]


class uniform:
    def __init__(self, xGrid, yGrid, zGrid, decomp):
        self.type = "uniform"
        self.device = decomp.device
        self.prec = decomp.prec
        self.dtypeNumpy = decomp.dtypeNumpy
        self.Nx, self.Ny, self.Nz = len(xGrid) - 1, len(yGrid) - 1, len(zGrid) - 1
        self.Lx = xGrid[-1] - xGrid[0]
        self.Ly = yGrid[-1] - yGrid[0]
        self.Lz = zGrid[-1] - zGrid[0]
        self.dx = self.Lx / float(self.Nx); self.dxi = 1.0 / self.dx
        self.dy = self.Ly / float(self.Ny); self.dyi = 1.0 / self.dy
        self.dz = self.Lz / float(self.Nz); self.dzi = 1.0 / self.dz
        for a in ("nover", "nxo_", "nx_", "nyo_", "ny_", "nzo_", "nz_", "imino_",
                  "jmino_", "kmino_", "imaxo_", "jmaxo_", "kmaxo_", "imin_",
                  "imax_", "jmin_", "jmax_", "kmin_", "kmax_"):
            setattr(self, a, getattr(decomp, a))

    @property
    def spacing(self):
        return (self.dx, self.dy, self.dz)


def Geometry_Base(IC, xGrid, yGrid, zGrid, decomp):
    return uniform(xGrid, yGrid, zGrid, decomp)
