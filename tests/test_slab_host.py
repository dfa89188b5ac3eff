"""Host logic of the x-slab decomposition (pyflow_b200.slab), on the CPU:
the plane split against the reference's formula, the periodic extension of
a global field, the ghost exchange and gather of both transports --
LocalSlabs in one process and DistSlabs over gloo with world sizes 2 and 3
-- against the periodic extension, and one shared restart file written and
read by the ranks' blocks.  No kernel runs here."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _ref_split(nx, npx, iproc):
    """The reference's x split, src/library/parallel.py:226-235."""
    q, r = nx // npx, nx % npx
    if iproc + 1 <= r:
        return iproc * (q + 1), q + 1
    return r * (q + 1) + (iproc - r) * q, q


@pytest.mark.parametrize("nx,npx", [(16, 1), (16, 2), (17, 3), (64, 8), (30, 7)])
def test_plane_ranges_match_reference_split(nx, npx):
    from pyflow_b200.slab import plane_ranges
    got = plane_ranges(nx, npx)
    assert got == [_ref_split(nx, npx, i) for i in range(npx)]
    assert sum(n for _, n in got) == nx


def test_plane_ranges_rejects_too_many_ranks():
    from pyflow_b200.slab import plane_ranges
    with pytest.raises(ValueError):
        plane_ranges(3, 4)


def _global(nx=13, ny=3, nz=4):
    return torch.arange(nx * ny * nz, dtype=torch.float64).reshape(nx, ny, nz)


def test_extend_fills_ghosts_periodically():
    from pyflow_b200.slab import extend
    g = _global()
    e = extend(g, 11, 2, halo=4)
    assert e.shape == (10, 3, 4)
    for a in range(10):
        assert torch.equal(e[a], g[(11 - 4 + a) % 13])


@pytest.mark.parametrize("R,planes", [(1, 4), (2, 1), (3, 4), (3, 2)])
def test_local_exchange_equals_periodic_extension(R, planes):
    from pyflow_b200.slab import HALO, LocalSlabs, extend, plane_ranges
    g = _global(14)
    rng = plane_ranges(14, R)
    # interiors from the global field, ghosts poisoned
    fields = []
    for x0, n in rng:
        e = torch.full((n + 2 * HALO, 3, 4), -1.0, dtype=torch.float64)
        e[HALO:HALO + n] = g[x0:x0 + n]
        fields.append([e, e.clone() * 2])
    LocalSlabs(R).exchange(fields, [n for _, n in rng], planes)
    for (x0, n), (a, b) in zip(rng, fields):
        want = extend(g, x0, n)
        lo, hi = HALO - planes, HALO + n + planes
        assert torch.equal(a[lo:hi], want[lo:hi])
        assert torch.equal(b[lo:hi], 2 * want[lo:hi])
        # planes beyond the exchanged depth are untouched
        assert bool((a[:lo] == -1.0).all()) and bool((a[hi:] == -1.0).all())


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _dist_worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from pyflow_b200.slab import HALO, DistSlabs, extend, plane_ranges
        T = DistSlabs()
        nx = 4 * world + 3
        g = _global(nx)
        x0, n = plane_ranges(nx, world)[rank]
        e = torch.full((n + 2 * HALO, 3, 4), -1.0, dtype=torch.float64)
        e[HALO:HALO + n] = g[x0:x0 + n]
        T.exchange([[e]], [n], HALO)
        ok_x = torch.equal(e, extend(g, x0, n))
        send = torch.tensor([float(rank), 10.0 * rank], dtype=torch.float64)
        recv = torch.zeros(2 * world, dtype=torch.float64)
        T.allgather([send], [recv])
        want = torch.tensor([v for r in range(world) for v in (float(r), 10.0 * r)],
                            dtype=torch.float64)
        q.put((rank, bool(ok_x), bool(torch.equal(recv, want))))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(180)
@pytest.mark.parametrize("world", [2, 3])
def test_dist_exchange_and_gather_gloo(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_dist_worker, args=(r, world, port, q)) for r in range(world)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(150)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=5) for _ in range(world))
    assert got == [(r, True, True) for r in range(world)]


def _io_worker(rank, world, port, path, q):
    """Each rank writes its slab's block of two variables into one shared
    restart file (file order computed on the host here, as the device
    transpose gives it), then reads its extended block back."""
    import numpy as np
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import pyflow_b200.dataReader as R
        from pyflow_b200.slab import HALO, plane_ranges
        nx, ny, nz = 4 * world + 5, 3, 4
        glob = [np.arange(nx * ny * nz, dtype=np.float64).reshape(nx, ny, nz) * (v + 1)
                for v in range(2)]
        x0, nxl = plane_ranges(nx, world)[rank]
        if rank == 0:
            with open(path, "wb") as f:
                f.write(R._header(nx, ny, nz, ["U", "V"], 0.1, 2.5))
                f.truncate(32 + 16 + 2 * 8 * nx * ny * nz)
        dist.barrier()
        view = R._fields_view(path, nx, ny, nz, 2, "r+")
        for v in range(2):
            block = np.ascontiguousarray(glob[v][x0:x0 + nxl].transpose(2, 1, 0))
            R.slab_block_write(view, v, x0, block)
        view.flush()
        del view
        dist.barrier()
        view = R._fields_view(path, nx, ny, nz, 2, "r")
        ok = True
        for v in range(2):
            got = R.slab_block_read(view, v, x0, nxl, HALO).transpose(2, 1, 0)
            want = np.pad(glob[v], ((HALO, HALO), (0, 0), (0, 0)), mode="wrap")[
                x0:x0 + nxl + 2 * HALO]
            ok = ok and np.array_equal(got, want)
        q.put((rank, bool(ok)))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(180)
@pytest.mark.parametrize("world", [2, 3])
def test_slab_restart_shared_file_gloo(world, tmp_path):
    """One restart file written by every rank's block (the layout of the
    reference's MPI-IO restart path) reads back with the serial reader, and
    each rank's periodic extended block reads back from it."""
    import numpy as np
    import pyflow_b200.dataReader as R
    path = str(tmp_path / "restart")
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_io_worker, args=(r, world, port, path, q)) for r in range(world)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(150)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=5) for _ in range(world))
    assert got == [(r, True) for r in range(world)]
    names, time, data = R.readNGArestart(path, headerOnly=False)
    nx = 4 * world + 5
    assert names == ["U", "V"] and time == 2.5
    for v in range(2):
        want = np.arange(nx * 3 * 4, dtype=np.float64).reshape(nx, 3, 4) * (v + 1)
        assert np.array_equal(data[..., v], want)
