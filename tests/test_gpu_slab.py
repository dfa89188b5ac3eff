"""The x-slab decomposition on one GPU (LocalSlabs: the ranks' slabs in one
process, exchanges as device copies, the same kernels and phases a rank runs
under DistSlabs).

* The predictor on slabs extended by four exchanged ghost planes is bitwise
  the predictor on the whole box (the slab interiors, gathered).
* A decomposed step (FP64, the reference's BiCGStab with reductions gathered
  across slabs) against the single-box pf_forward_step: the solves reduce in
  a different order and form rho1 differently, so they agree to the solver
  tolerance -- velocity and pressure to 1e-8 of their largest value after
  three steps, iteration counts within 10 % per step (BiCGStab's count at a
  1e-10 tolerance moves by a few iterations with the rounding of its
  scalars).
* Different slab counts give the same fields to 1e-9 (only the reductions'
  order differs, which may move the stop by an iteration).
* The divergence left by a decomposed step is as small as the single-box
  step's."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _fields(shape, seed=3):
    import pyflow_b200.initial as ic
    return [torch.tensor(a, device="cuda") for a in ic.spectral_velocity(shape, k0=3.0, seed=seed)]


@pytest.mark.parametrize("R,shape", [(1, (16, 12, 16)), (2, (16, 12, 16)), (3, (20, 12, 16)),
                                     (4, (19, 8, 12))])
def test_slab_predictor_bitwise(R, shape):
    import pyflow_b200.ops as ops
    from pyflow_b200.slab import LocalSlabs, SlabDomain
    sp = tuple(2 * np.pi / n for n in shape)
    u, v, w = _fields(shape)
    D = SlabDomain(shape, sp, 0.01, 1.0, 0.004, LocalSlabs(R))
    D.set_state(u, v, w)
    D._xchg(["u", "v", "w"], 4)
    for s in D.slabs:
        ops.predictor_step(s.u, s.v, s.w, sp, 0.01, 1.0, 0.004)
    ops.predictor_step(u, v, w, sp, 0.01, 1.0, 0.004)
    torch.cuda.synchronize()
    for name, ref in (("u", u), ("v", v), ("w", w)):
        assert torch.equal(D.gather(name), ref), name


def _single(shape, sp, nu, dt, steps, f0):
    import pyflow_b200.ops as ops
    a = [t.clone() for t in f0] + [torch.zeros_like(f0[0]), torch.zeros_like(f0[0])]
    its = []
    for _ in range(steps):
        info = ops.forward_step(*a, sp, nu, 1.0, dt, min_res=1e-10, max_it=5000)
        its.append(info.iterations)
    return a, its


def _slabs(shape, sp, nu, dt, steps, f0, R):
    from pyflow_b200.slab import LocalSlabs, SlabDomain
    D = SlabDomain(shape, sp, nu, 1.0, dt, LocalSlabs(R), min_res=1e-10, max_it=5000, poll=1)
    D.set_state(*f0)
    infos = [D.forward_step() for _ in range(steps)]
    return D, infos


@pytest.mark.parametrize("R,shape", [(2, (24, 16, 20)), (3, (26, 16, 16))])
def test_slab_step_matches_single_box(R, shape):
    sp = tuple(2 * np.pi / n for n in shape)
    nu, dt, steps = 0.01, 0.005, 3
    f0 = _fields(shape, seed=11)
    a, its = _single(shape, sp, nu, dt, steps, f0)
    D, infos = _slabs(shape, sp, nu, dt, steps, f0, R)
    torch.cuda.synchronize()
    for info, it in zip(infos, its):
        assert info.status == 0 and info.max_res <= 1e-10
        assert abs(info.iterations - it) <= max(2, 0.1 * it), (info.iterations, it)
    for name, ref in zip(("u", "v", "w", "p"), a[:4]):
        got = D.gather(name)
        err = (got - ref).abs().max().item()
        assert err <= 1e-8 * ref.abs().max().item(), (name, err)
    import pyflow_b200.ops as ops
    div_slab = ops.div_vel(D.gather("u"), D.gather("v"), D.gather("w"), sp).abs().max().item()
    div_one = ops.div_vel(*a[:3], sp).abs().max().item()
    assert div_slab <= 10 * div_one + 1e-12


def test_slab_counts_agree():
    shape = (24, 16, 16)
    sp = tuple(2 * np.pi / n for n in shape)
    f0 = _fields(shape, seed=12)
    outs = []
    for R in (1, 2, 4):
        D, _ = _slabs(shape, sp, 0.01, 0.005, 2, f0, R)
        outs.append([D.gather(n) for n in ("u", "v", "w")])
    torch.cuda.synchronize()
    for other in outs[1:]:
        for x, y in zip(outs[0], other):
            assert (x - y).abs().max().item() <= 1e-9 * y.abs().max().item()


def test_slab_zero_source_stops_at_once():
    """A divergence-free field with nothing to correct: the first gamma is
    zero, the reference's loop breaks (src/solver/pressure.py:247-248) and
    the step leaves the predicted field; every slab reports the same."""
    from pyflow_b200.slab import LocalSlabs, SlabDomain
    shape = (12, 8, 8)
    sp = tuple(2 * np.pi / n for n in shape)
    z = torch.zeros(shape, dtype=torch.float64, device="cuda")
    D = SlabDomain(shape, sp, 0.01, 1.0, 0.005, LocalSlabs(2), poll=1)
    D.set_state(z, z, z)
    info = D.forward_step()
    assert info.iterations == 0 and info.max_res == 0.0
    assert float(D.gather("u").abs().max()) == 0.0


def test_slab_restart_round_trip(tmp_path):
    """writeNGArestart_slabs from three slabs gives the file the serial writer
    gives for the whole box (read back by the serial reader), and
    readNGArestart_slabs fills every slab's interior and ghost planes."""
    import pyflow_b200.dataReader as R
    from pyflow_b200.slab import LocalSlabs, SlabDomain, extend
    shape = (20, 12, 16)
    sp = tuple(2 * np.pi / n for n in shape)
    f = _fields(shape, seed=4) + [torch.randn(shape, dtype=torch.float64, device="cuda")]
    D = SlabDomain(shape, sp, 0.01, 1.0, 0.005, LocalSlabs(3))
    D.set_state(*f)
    path = str(tmp_path / "restart_slabs")
    R.writeNGArestart_slabs(path, D, dt=0.005, time=1.25)
    names, time, data = R.readNGArestart(path, headerOnly=False)
    assert names == ["U", "V", "W", "P"] and time == 1.25
    for v, a in enumerate(f):
        assert np.array_equal(data[..., v], a.cpu().numpy())
    E = SlabDomain(shape, sp, 0.01, 1.0, 0.005, LocalSlabs(3))
    assert R.readNGArestart_slabs(path, E) == 1.25
    for s in E.slabs:
        for name, a in zip(("u", "v", "w", "p"), f):
            assert torch.equal(getattr(s, name), extend(a, s.x0, s.nxl))
