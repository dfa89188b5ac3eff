"""The x-slab solve protocol across processes, on the host.

The phases of the distributed BiCGStab (csrc/pf_slab.cu: init, START / NEXT,
APPLY_P, S, APPLY_S, FINAL, each fold of the gathered sums in rank order)
are restated here in numpy, as test infrastructure; the ranks are gloo
processes that exchange ghost planes and gather their 2-double partial sums
through the product's transport (slab.DistSlabs), in the order SlabDomain.solve
uses.  The decomposed solve must reach the oracle's single-box BiCGStab
(the reference's algorithm, src/solver/pressure.py:196-297) to the solver
tolerance, and every rank must stop at the same iteration with the same
status -- the property that keeps the ranks' collective sequences identical.
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _lap_interior(A, H, nxl, c):
    """Pressure_Base.applyOperator on the interior planes of an extended
    array (x neighbours from the planes beside it, y and z periodic), terms
    in the kernels' order."""
    I = slice(H, H + nxl)
    a = A[I]
    b = np.zeros_like(a)
    b += A[H - 1:H - 1 + nxl] * c[0][0]
    b += a * c[0][1]
    b += A[H + 1:H + 1 + nxl] * c[0][2]
    b += np.roll(a, 1, 1) * c[1][0]
    b += a * c[1][1]
    b += np.roll(a, -1, 1) * c[1][2]
    b += np.roll(a, 1, 2) * c[2][0]
    b += a * c[2][1]
    b += np.roll(a, -1, 2) * c[2][2]
    return b


def _solve_rank(T, div_int, spacing, rho, dt, min_res, max_it, H):
    """One rank's decomposed solve: returns (DP interior, iterations, status,
    max_res)."""
    nxl, ny, nz = div_int.shape
    dx, dy, dz = spacing
    vol = (dx * dy) * dz
    c = [[(d * d) * (-1.0 * vol), ((-2.0 * d) * d) * (-1.0 * vol), (d * d) * (-1.0 * vol)]
         for d in (1.0 / dx, 1.0 / dy, 1.0 / dz)]
    shape = (nxl + 2 * H, ny, nz)
    I = slice(H, H + nxl)
    res, res0, pp, vv, s, t, DP = (np.zeros(shape) for _ in range(7))
    res[I] = (div_int * (rho / dt)) * (-1.0 * vol)
    res0[I] = res[I]
    world = T.size

    def gather(a, b):
        send = torch.tensor([a, b], dtype=torch.float64)
        recv = torch.zeros(2 * world, dtype=torch.float64)
        T.allgather([send], [recv])
        r = recv.numpy().reshape(world, 2)
        return r

    def xchg(f):
        tf = torch.from_numpy(f)
        T.exchange([[tf]], [nxl], 1, halo=H)

    r = gather(float((res[I] * res0[I]).sum()), float(np.abs(res[I]).max()))
    max_res0 = max(r[:, 1])
    rho1 = 0.0
    for q in range(world):
        rho1 += r[q, 0]
    rho2, alpha, omega = 1.0, 0.0, 1.0
    it, status, max_res = 0, 0, 0.0
    while True:
        beta = alpha * rho1 / (rho2 * omega)
        pp[I] = (pp[I] - omega * vv[I]) * beta + res[I]
        xchg(pp)
        vv[I] = _lap_interior(pp, H, nxl, c)
        r = gather(float((vv[I] * res0[I]).sum()), 0.0)
        gamma = 0.0
        for q in range(world):
            gamma += r[q, 0]
        if gamma == 0.0:
            status = 3
            break
        alpha = rho1 / gamma
        DP[I] += alpha * pp[I]
        s[I] = res[I] - alpha * vv[I]
        xchg(s)
        t[I] = _lap_interior(s, H, nxl, c)
        r = gather(float((s[I] * t[I]).sum()), float((t[I] * t[I]).sum()))
        b1 = b2 = 0.0
        for q in range(world):
            b1 += r[q, 0]
            b2 += r[q, 1]
        if b2 == 0.0:
            status = 3
            break
        omega = b1 / b2
        DP[I] += omega * s[I]
        res[I] = s[I] - omega * t[I]
        r = gather(float((res[I] * res0[I]).sum()), float(np.abs(res[I]).max()))
        rho2 = rho1
        rho1 = 0.0
        for q in range(world):
            rho1 += r[q, 0]
        max_res = max(r[:, 1]) / max_res0
        it += 1
        if max_res <= min_res:
            break
        if it >= max_it:
            status = 4
            break
    return DP[I].copy(), it, status, max_res


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import oracle as O
        from pyflow_b200.slab import HALO, DistSlabs, plane_ranges
        shape = (4 * world + 6, 8, 10)
        sp = (2 * np.pi / shape[0], 0.7, 0.55)
        rng = np.random.default_rng(21)
        u, v, w = (rng.standard_normal(shape) for _ in range(3))
        div = O.div_vel(sp, u, v, w)
        x0, nxl = plane_ranges(shape[0], world)[rank]
        DP, it, status, max_res = _solve_rank(DistSlabs(), div[x0:x0 + nxl], sp, 1.0, 0.01,
                                              1e-10, 2000, HALO)
        parts = [None] * world
        dist.all_gather_object(parts, (x0, DP, it, status))
        if rank == 0:
            DP_all = np.concatenate([p[1] for p in sorted(parts, key=lambda p: p[0])])
            ref = O.bicgstab(sp, div, np.zeros(shape), 1.0, 0.01, 1e-10, 2000)
            err = float(np.abs(DP_all - ref[0]).max() / np.abs(ref[0]).max())
            q.put(("result", err, [p[2] for p in parts], [p[3] for p in parts], ref[3],
                   max_res))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(240)
@pytest.mark.parametrize("world", [2, 3])
def test_decomposed_solve_over_gloo_matches_oracle(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(200)
        assert p.exitcode == 0
    tag, err, its, statuses, ref_its, max_res = q.get(timeout=5)
    assert tag == "result"
    # every rank stopped at the same iteration with the same status
    assert len(set(its)) == 1 and statuses == [0] * world, (its, statuses)
    assert max_res <= 1e-10
    assert abs(its[0] - ref_its) <= max(2, 0.1 * ref_its), (its[0], ref_its)
    assert err <= 1e-8, err
