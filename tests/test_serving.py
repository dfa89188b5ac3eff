"""Serving loop: host logic on CPU (request stream, percentiles, footprint),
continuous batching and admission on the GPU."""
import numpy as np
import pytest
import torch


def test_percentile_and_stream():
    import pyflow_b200.serving as S
    assert S.percentile([1, 2, 3, 4], 50) == 2.5
    assert S.percentile(list(range(101)), 99) == 99
    reqs = S.stream_requests(600, rate=10.0)
    assert {r.n for r in reqs} == {32, 48, 64, 96, 128, 192}
    arr = np.array([r.arrival for r in reqs])
    assert np.all(np.diff(arr) >= 0) and abs(np.mean(np.diff(arr)) - 0.1) < 0.02
    assert all(abs(r.nu - 0.02 * 32 / r.n) < 1e-15 and r.seed == 1000 + r.id for r in reqs)


def test_footprint_grows_with_grid():
    import pyflow_b200.serving as S
    a, b = S.footprint_bytes(32), S.footprint_bytes(64)
    assert b > 7 * a and a > 5 * 8 * 32 ** 3


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["mixed_mg", "fp64"])
def test_results_same_alone_and_in_mix(prec):
    """Batched serving: each request's fields after its steps are bitwise the
    same served alone, in a mix of sizes arriving over time (batch graphs
    rebuilt as requests join and leave), and with one graph per request."""
    import pyflow_b200.serving as S
    sizes = [16, 24, 32, 16, 64, 20, 48]
    reqs = [S.Request(id=i, n=n, seed=1000 + i, nu=0.02 * 32 / n, dt=0.01, steps=4 + i % 3,
                      arrival=0.002 * i) for i, n in enumerate(sizes)]
    alone = {}
    for r in reqs:
        srv = S.Server(max_slots=1, prec=prec, keep_fields=True)
        res = srv.run([S.Request(**{**r.__dict__, "arrival": 0.0})])
        assert res[0].status == "ok", res[0]
        alone[r.id] = res[0]
    srv = S.Server(max_slots=4, prec=prec, keep_fields=True)
    mixed = srv.run(reqs)
    assert srv.max_active > 1 and srv.rebuilds > 2
    streams = S.Server(max_slots=4, prec=prec, keep_fields=True, batched=False).run(reqs)
    assert len(mixed) == len(reqs) == len(streams)
    by_stream = {r.id: r for r in streams}
    for m in mixed:
        a = alone[m.id]
        assert m.status == "ok"
        for x, y, z in zip(m.fields, a.fields, by_stream[m.id].fields):
            assert torch.equal(x, y) and torch.equal(x, z)
        assert m.stats["max_res"] <= 1e-10
        assert m.stats["steps"] == m.steps


@pytest.mark.gpu
def test_batch_plan_matches_step_plans():
    """One BatchPlan over requests of different sizes advances each exactly
    like its own StepPlan (grouped RK4 stages, branch-parallel solves)."""
    import pyflow_b200.initial as ic
    from pyflow_b200.plan import BatchPlan, Member, StepPlan
    shapes = [(32, 32, 32), (24, 20, 28), (64, 64, 64), (16, 48, 32)]
    ref, members = [], []
    for i, sh in enumerate(shapes):
        sp = tuple(2 * np.pi / n for n in sh)
        f0 = [torch.tensor(a, device="cuda") for a in ic.spectral_velocity(sh, seed=i)]
        fa = [t.clone() for t in f0] + [torch.zeros_like(f0[0]) for _ in range(2)]
        fb = [t.clone() for t in f0] + [torch.zeros_like(f0[0]) for _ in range(2)]
        pl = StepPlan(*fa, sp, 0.01, 1.0, 0.004, prec="mixed_mg")
        pl.launch(3)
        torch.cuda.synchronize()
        ref.append((fa, pl.stats()))
        pl.close()
        members.append(Member(*fb, sp, 0.01, 1.0, 0.004, prec="mixed_mg"))
    bp = BatchPlan(members)
    bp.launch(2)
    bp2 = BatchPlan(members[::-1])      # a rebuilt batch carries the state over
    bp2.launch(1)
    torch.cuda.synchronize()
    for (fa, st), m in zip(ref, members):
        for x, y in zip(fa[:4], m.fields[:4]):
            assert torch.equal(x, y)
        got = m.stats()
        for k in ("max_u", "tke", "max_div", "max_res", "iterations", "total_iterations",
                  "steps"):
            assert got[k] == st[k], k
    bp.close()
    bp2.close()


@pytest.mark.gpu
def test_admission_by_free_memory():
    import pyflow_b200.serving as S
    one = S.footprint_bytes(24)
    reqs = [S.Request(id=i, n=24, seed=1000 + i, nu=0.02, dt=0.01, steps=2) for i in range(4)]
    reqs.append(S.Request(id=9, n=64, seed=7, nu=0.01, dt=0.01, steps=2))
    # a fake free-HBM provider with room for exactly one 24^3 request
    srv = S.Server(max_slots=8, free_hbm=lambda used: int(1.5 * one) - used, prec="fp64")
    res = srv.run(reqs)
    by = {r.id: r for r in res}
    assert srv.max_active == 1
    assert all(by[i].status == "ok" for i in range(4))
    assert by[9].status == "rejected"


def test_assign_requests_balances_and_rejects():
    import pyflow_b200.serving as S
    reqs = S.stream_requests(64, rate=20.0)
    big = S.footprint_bytes(192)
    shards, rej = S.assign_requests(reqs, [10 * big, 10 * big, S.footprint_bytes(64)])
    ids = sorted(r.id for sh in shards for r in sh)
    assert ids == sorted(r.id for r in reqs) and not rej
    # the small rank only ever gets grids that fit it
    assert all(r.n <= 64 for r in shards[2])
    work = [sum(r.n ** 3 * r.steps for r in sh) for sh in shards[:2]]
    assert max(work) <= 1.5 * min(work)
    _, rej = S.assign_requests(reqs, [S.footprint_bytes(48)])
    assert {r.n for r in rej} == {64, 96, 128, 192}


def _shard_worker(rank, world, port, q):
    import torch.distributed as dist
    import pyflow_b200.serving as S
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank,
                            world_size=world)
    try:
        reqs = S.stream_requests(40, rate=10.0)
        free = [8 * S.footprint_bytes(192)] * world
        shards, _ = S.assign_requests(reqs, free)
        mine = [r.id for r in shards[rank]]
        allv = [None] * world
        dist.all_gather_object(allv, mine)
        work = torch.tensor([float(sum(r.n ** 3 * r.steps for r in shards[rank]))],
                            dtype=torch.float64)
        dist.all_reduce(work)
        q.put((rank, allv, float(work.item()),
               float(sum(r.n ** 3 * r.steps for r in reqs))))
    finally:
        dist.destroy_process_group()


def test_request_sharding_two_ranks_gloo():
    """Two ranks compute the same assignment independently: their shards are
    disjoint, cover the stream, and the aggregate work sums to the total."""
    import socket
    import torch.multiprocessing as mp
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_shard_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, allv, work, total in out:
        a, b = allv
        assert not set(a) & set(b) and sorted(a + b) == list(range(40))
        assert work == total
