"""NGA config / restart files (format of src/data/dataReader.py:60-208).

The restart format is a header ``<4i nx,ny,nz,nvar><2d dt,time><8-char names>``
followed by each variable in Fortran order (float64).

* ``readNGArestart`` / ``writeNGArestart``: serial numpy, host arrays.
* ``readNGArestart_device`` / ``writeNGArestart_device``: straight between
  the file and device fields (the reference's checkpoint path is MPI-IO from
  host copies, src/data/dataReader.py:215-390).  Each field is transposed to
  or from the file's order on the device (pf_restart_pack / _unpack), then
  moves in chunks through two pinned host buffers: the device-to-host copy
  of chunk k+1 (a copy stream) overlaps the file write of chunk k (a writer
  thread), and reading overlaps the same way.  No whole-field host copy.
PyFlow.run reads its initial state and writes its checkpoints this way.
"""
import ctypes
import struct
import threading

import numpy as np

CHUNK_BYTES = 1 << 26   # 64 MiB per pinned staging buffer


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


def _header(nx, ny, nz, names, dt, time):
    out = struct.pack("<4i", nx, ny, nz, len(names)) + struct.pack("<2d", dt, time)
    for n in names:
        out += n.ljust(8)[:8].encode()
    return out


def _lib():
    from . import _lib as L
    return L


def writeNGArestart_device(fName, fields, names, dt, time, chunk_bytes=CHUNK_BYTES):
    """Write device FP64 fields (each (nx, ny, nz), C order) as a restart
    file, straight from device memory."""
    import torch
    from . import ops
    L = _lib()
    nx, ny, nz = fields[0].shape
    dev = fields[0].device
    g = ops.grid((nx, ny, nz), (1.0, 1.0, 1.0))
    n = nx * ny * nz
    scratch = torch.empty(n, dtype=torch.float64, device=dev)
    per = max(1, min(n, chunk_bytes // 8))
    pinned = [torch.empty(per, dtype=torch.float64).pin_memory() for _ in range(2)]
    copy = torch.cuda.Stream(dev)
    events = [torch.cuda.Event() for _ in range(2)]
    main = torch.cuda.current_stream(dev)
    with open(fName, "wb") as f:
        f.write(_header(nx, ny, nz, names, dt, time))
        for a in fields:
            ops._check(a, (nx, ny, nz), torch.float64, "field")
            L.check("pf_restart_pack", L.lib().pf_restart_pack(
                ctypes.byref(g), ops._p(a), ops._p(scratch), ctypes.c_void_p(main.cuda_stream)))
            copy.wait_stream(main)
            writer, k = None, 0
            for s0 in range(0, n, per):
                m = min(per, n - s0)
                buf = pinned[k & 1]
                with torch.cuda.stream(copy):
                    buf[:m].copy_(scratch[s0:s0 + m], non_blocking=True)
                events[k & 1].record(copy)
                if writer is not None:
                    writer.join()
                events[k & 1].synchronize()
                view = buf[:m].numpy()
                writer = threading.Thread(target=f.write, args=(memoryview(view).cast("B"),))
                writer.start()
                k += 1
            if writer is not None:
                writer.join()
    # the scratch buffer is free once the copies have finished
    copy.synchronize()


def readNGArestart_device(fName, device, nvar=None, chunk_bytes=CHUNK_BYTES):
    """(names, time, [fields]) of a restart file, each field a device FP64
    tensor (nx, ny, nz) read straight into device memory."""
    import torch
    from . import ops
    L = _lib()
    (nx, ny, nz, nv), dt, time = readNGArestart_dims(fName)
    names = readNGArestart(fName, headerOnly=True)[0]
    nv = nv if nvar is None else min(nv, nvar)
    dev = torch.device(device)
    g = ops.grid((nx, ny, nz), (1.0, 1.0, 1.0))
    n = nx * ny * nz
    per = max(1, min(n, chunk_bytes // 8))
    pinned = [torch.empty(per, dtype=torch.float64).pin_memory() for _ in range(2)]
    done = [torch.cuda.Event() for _ in range(2)]
    copy = torch.cuda.Stream(dev)
    main = torch.cuda.current_stream(dev)
    scratch = torch.empty(n, dtype=torch.float64, device=dev)
    out = []
    k = 0   # chunks so far (over all variables): buffer k & 1 was used by chunk k - 2
    with open(fName, "rb") as f:
        f.seek(32 + 8 * len(names))
        for _ in range(nv):
            copy.wait_stream(main)          # the scratch buffer is free
            for s0 in range(0, n, per):
                m = min(per, n - s0)
                buf = pinned[k & 1]
                if k >= 2:
                    done[k & 1].synchronize()   # its previous copy has left
                f.readinto(memoryview(buf[:m].numpy()).cast("B"))
                with torch.cuda.stream(copy):
                    scratch[s0:s0 + m].copy_(buf[:m], non_blocking=True)
                done[k & 1].record(copy)
                k += 1
            main.wait_stream(copy)
            field = torch.empty((nx, ny, nz), dtype=torch.float64, device=dev)
            L.check("pf_restart_unpack", L.lib().pf_restart_unpack(
                ctypes.byref(g), ops._p(scratch), ops._p(field),
                ctypes.c_void_p(main.cuda_stream)))
            out.append(field)
    main.synchronize()
    return names[:nv], time, out


# --------------------------------------------------------------------------
# One shared restart file for an x-slab decomposition (slab.SlabDomain): the
# counterpart of the reference's MPI-IO restart path
# (src/data/dataReader.py:215-390), where every rank writes and reads its own
# part of one file.  In the file's Fortran order a rank's planes
# [x0, x0 + nxl) are, for every (j, k), a run of nxl values, so the file's
# variables are viewed as [nvar][nz][ny][nx] arrays and a rank reads or
# writes the x range of its slab.

def _fields_view(fName, nx, ny, nz, nvar, mode):
    return np.memmap(fName, dtype="<f8", mode=mode, offset=32 + 8 * nvar,
                     shape=(nvar, nz, ny, nx))


def slab_block_write(view, var, x0, block):
    """Store ``block`` ([nz][ny][nxl], file order) as planes x0 .. x0 + nxl
    of variable ``var``."""
    view[var, :, :, x0:x0 + block.shape[2]] = block


def slab_block_read(view, var, x0, nxl, halo):
    """Planes x0 - halo .. x0 + nxl + halo (periodic) of variable ``var`` in
    file order, [nz][ny][nxl + 2 halo]."""
    nx = view.shape[3]
    ix = (np.arange(nxl + 2 * halo) + (x0 - halo)) % nx
    return np.ascontiguousarray(view[var][:, :, ix])


def writeNGArestart_slabs(fName, D, names=("U", "V", "W", "P"), dt=0.0, time=0.0,
                          barrier=None):
    """Write the fields of a slab.SlabDomain ``D`` into one restart file.
    Every process holding slabs calls it with the same arguments; a
    barrier separates the header from the ranks' writes and ends the call
    once every rank has written (``barrier``; by default the process group's
    barrier when the slabs are spread over processes).  Each
    slab's interior is transposed to the file's order on the device
    (pf_restart_pack) and written as the runs of its x range."""
    import torch
    from . import ops
    from .slab import HALO
    L = _lib()
    nx, ny, nz = D.shape
    fields = [n.lower() for n in names]
    if barrier is None and len(D.slabs) < D.T.size:
        import torch.distributed as dist
        group = getattr(D.T, "group", None)
        barrier = lambda: dist.barrier(group)  # noqa: E731
    first = D.slabs[0].x0 == 0
    if first:
        with open(fName, "wb") as f:
            f.write(_header(nx, ny, nz, list(names), dt, time))
            f.truncate(32 + 8 * len(names) + 8 * nx * ny * nz * len(names))
    if barrier is not None:
        barrier()
    view = _fields_view(fName, nx, ny, nz, len(names), "r+")
    for s in D.slabs:
        g = ops.grid((s.nxl, ny, nz), (1.0, 1.0, 1.0))
        scratch = torch.empty(s.nxl * ny * nz, dtype=torch.float64, device=s.u.device)
        for v, name in enumerate(fields):
            interior = getattr(s, name)[HALO:HALO + s.nxl]
            L.check("pf_restart_pack", L.lib().pf_restart_pack(
                ctypes.byref(g), ops._p(interior), ops._p(scratch), ops._stream(interior)))
            slab_block_write(view, v, s.x0, scratch.cpu().numpy().reshape(nz, ny, s.nxl))
    view.flush()
    del view
    if barrier is not None:
        barrier()


def readNGArestart_slabs(fName, D, names=("U", "V", "W", "P")):
    """Fill the held slabs of ``D`` (interior and ghost planes) from one
    restart file: each slab reads the periodic x range of its extended array
    and transposes it on the device (pf_restart_unpack).  Returns the file's
    time."""
    import torch
    from . import ops
    from .slab import HALO
    L = _lib()
    (nx, ny, nz, nv), dt, time = readNGArestart_dims(fName)
    if (nx, ny, nz) != tuple(D.shape):
        raise ValueError("restart grid %s does not match the domain %s" % ((nx, ny, nz), D.shape))
    file_names = readNGArestart(fName, headerOnly=True)[0]
    view = _fields_view(fName, nx, ny, nz, nv, "r")
    h = HALO
    for s in D.slabs:
        ne = s.nxl + 2 * h
        g = ops.grid((ne, ny, nz), (1.0, 1.0, 1.0))
        for name in names:
            v = file_names.index(name)
            block = torch.from_numpy(slab_block_read(view, v, s.x0, s.nxl, h)).to(s.u.device)
            dst = getattr(s, name.lower())
            L.check("pf_restart_unpack", L.lib().pf_restart_unpack(
                ctypes.byref(g), ops._p(block), ops._p(dst), ops._stream(dst)))
        s.DP.zero_()
    torch.cuda.synchronize()
    del view
    return time
