"""Generate golden fixtures by running the unmodified reference PyFlow.

Run in a container that has the reference source tree, naming its root in
PF_REFERENCE_ROOT (required; the directory that holds the reference's src/):

    PF_REFERENCE_ROOT=<reference checkout> python tests/golden/make_golden.py

Writes ``tests/golden/*.npz``.  The fixtures pin the CPU oracle
(oracle/pf_oracle.c) to the reference, and the CUDA path to the oracle.  The
reference runs on CPU in FP64 through ref_harness.py's single-rank shims.

Fixtures
--------
ops_12x16x20.npz   per-operator cases on a non-cubic, anisotropic periodic box:
                   rhs_NavierStokes.evaluate with constant VISC and with a
                   variable VISC plus 'tensor' SFS stresses, div_vel,
                   applyOperator, RK4.step / Euler.step predictors,
                   solver_bicgstab.solve, vel_corr.
jacobi_16.npz      solver_jacobi.solve on a cubic 16^3 box (the reference's
                   Jacobi assumes dx = dy = dz).
sgs_12x16x20.npz   SGS closures on the same kind of box: Smagorinsky eddy
                   viscosity (stress_constCs.eddyVisc), gradient-model stresses
                   (residual_stress.update), and the RHS with each closure
                   active (VISC_P = mu + mu_t; 'tensor' stresses added).
adjoint_12x16x20.npz  the reference's adjoint RHS (rhs_adjPredictor.evaluate,
                   src/solver/adjoint.py:94-298) at a random state for a random
                   adjoint field, its ML-closure term zeroed by a stand-in model
                   that keeps the autograd graph; and one reference Euler
                   adjoint step (adjoint projection, then the adjoint advancer;
                   src/data/domain.py:409-438).
run_32.npz         PyFlow.run: 32^3 seeded spectral field (k0 = 4, urms = 1),
                   nu = 0.01, dt = 0.005, RK4 + BiCGStab to 1e-10, 5 steps:
                   final u, v, w, p and per-step max residual, iteration count
                   and monitor statistics.
ml_16.npz          rhs_NavierStokes.evaluate with the reference's 'source' ML
                   closure (sfsmodel_ML, a seeded random network whose
                   weights are stored in the fixture) on a 16^3 box, and the
                   closure's inputs as the RHS hands them over (ci).
finalize_8.npz     sfsmodel_ML.residual_stress.finalize over seven training
                   windows with seeded gradients (gradient averaging over
                   numSumDistr windows, RMSprop, learning-rate schedule).
target_12x16x20.npz  Domain.TargetDataVelCorr: projection of a random target
                   field (and the DP it adds to the simulation pressure).
run_64.npz         PyFlow.run of the 64^3 plain-DNS workload (seed 0, k0 = 4,
                   nu = 0.01, dt = 0.005, 20 RK4 steps): final u, v, w, p on
                   every 4th cell of each axis, their sum / sum of squares /
                   max, and the per-step residuals, iterations and statistics.
"""
import os
import sys
import types
import warnings

import numpy as np

warnings.filterwarnings("ignore")
HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, HERE)
sys.path.insert(0, REPO)

import ref_harness as H  # noqa: E402


def _state(ns, d, a):
    return ns.state.state_P(d, np.ascontiguousarray(a).copy())


def ops_case(out):
    import torch
    nx, ny, nz = 12, 16, 20
    lengths = (2 * np.pi, 2.1, 3.3)
    S = H.make_setup(nx, ny, nz, *lengths)
    ns, d = S.ns, S.decomp
    rng = np.random.default_rng(1234)
    # smooth-ish random fields: low-pass filtered noise plus white noise
    u, v, w = (rng.standard_normal((nx, ny, nz)) for _ in range(3))
    visc = 0.01 + 0.005 * rng.random((nx, ny, nz))
    sfs = [0.1 * rng.standard_normal((nx, ny, nz)) for _ in range(6)]
    mu, rho, dt = 0.01, 1.3, 2.0e-3
    res = dict(shape=np.array([nx, ny, nz]),
               spacing=np.array([S.geo.dx, S.geo.dy, S.geo.dz]),
               u=u, v=v, w=w, visc=visc, sfs=np.stack(sfs),
               mu=mu, rho=rho, dt=dt)

    class Blank:
        modelType = "eddyVisc"

    class Tensor:
        modelType = "tensor"

    # rhs with constant VISC (src/data/domain.py:130-131)
    VISC = torch.ones(nx + 4, ny + 4, nz + 4, dtype=torch.float64) * mu
    rhs = ns.velocity.rhs_NavierStokes(d, S.metric, rho, VISC, Blank())
    su, sv, sw = (_state(ns, d, a) for a in (u, v, w))
    rhs.evaluate(su, sv, sw)
    res["rhs_const"] = np.stack([rhs.rhs_u.numpy(), rhs.rhs_v.numpy(),
                                 rhs.rhs_w.numpy()])
    # rhs with variable VISC + tensor SFS
    m = Tensor()
    for nm, a in zip(["FXX", "FYY", "FZZ", "FXY", "FXZ", "FYZ"], sfs):
        setattr(m, nm, H.padded(d, a))
    rhs2 = ns.velocity.rhs_NavierStokes(d, S.metric, rho, H.padded(d, visc), m)
    rhs2.evaluate(su, sv, sw)
    res["rhs_visc_sfs"] = np.stack([rhs2.rhs_u.numpy(), rhs2.rhs_v.numpy(),
                                    rhs2.rhs_w.numpy()])
    # divergence and Laplacian
    dv = torch.zeros(nx, ny, nz, dtype=torch.float64)
    S.metric.div_vel(su, sv, sw, dv)
    res["div"] = dv.numpy().copy()
    P = ns.pressure.Pressure_Base(d, S.metric)
    B = torch.zeros(nx, ny, nz, dtype=torch.float64)
    P.applyOperator(H.padded(d, u), B)
    res["lap_u"] = B.numpy().copy()

    # RK4 and Euler predictors (constant VISC)
    class RHSSet:
        pass

    rs = RHSSet()
    rs.rhs1, rs.rhs2, rs.rhs3, rs.rhs4 = (
        ns.velocity.rhs_NavierStokes(d, S.metric, rho, VISC, Blank())
        for _ in range(4))
    su, sv, sw = (_state(ns, d, a) for a in (u, v, w))
    tu, tv, tw = (_state(ns, d, a) for a in (u, v, w))
    ns.advancer.RK4(su, tu, sv, tv, sw, tw, rs).step(dt)
    res["rk4"] = np.stack([su.interior().numpy(), sv.interior().numpy(),
                           sw.interior().numpy()])
    su, sv, sw = (_state(ns, d, a) for a in (u, v, w))
    ns.advancer.Euler(su, sv, sw, rs).step(dt)
    res["euler"] = np.stack([su.interior().numpy(), sv.interior().numpy(),
                             sw.interior().numpy()])

    # BiCGStab on the divergence of the RK4 predictor, then the projection
    pu, pv, pw = res["rk4"]
    su, sv, sw = (_state(ns, d, a) for a in (pu, pv, pw))
    src = torch.zeros(nx, ny, nz, dtype=torch.float64)
    S.metric.div_vel(su, sv, sw, src)
    res["bicg_source"] = src.numpy().copy()
    p0 = 0.1 * rng.standard_normal((nx, ny, nz))
    res["p0"] = p0
    sDP = _state(ns, d, np.zeros((nx, ny, nz)))
    sp = _state(ns, d, p0)
    iters = [0]
    orig = P.__class__.applyOperator

    def counting(self, A, Bo):
        iters[0] += 1
        return orig(self, A, Bo)

    solver = ns.pressure.solver_bicgstab(S.comms, d, S.metric, S.geo, rho, dt,
                                         1e-10, 500)
    solver.pressure.applyOperator = types.MethodType(counting, solver.pressure)
    r = solver.solve(sDP, sp, src)
    res["bicg_DP"] = sDP.interior().numpy().copy()
    res["bicg_p"] = sp.interior().numpy().copy()
    res["bicg_max_res"] = float(r)
    res["bicg_iters"] = iters[0] // 2
    S.metric.grad_P(sDP)
    su.vel_corr(sDP.grad_x, dt / rho)
    sv.vel_corr(sDP.grad_y, dt / rho)
    sw.vel_corr(sDP.grad_z, dt / rho)
    res["corr"] = np.stack([su.interior().numpy(), sv.interior().numpy(),
                            sw.interior().numpy()])
    np.savez_compressed(os.path.join(out, "ops_12x16x20.npz"), **res)
    print("ops: bicgstab iters", res["bicg_iters"], "max_res", r)


def sgs_case(out):
    import torch
    nx, ny, nz = 12, 16, 20
    lengths = (2 * np.pi, 2.1, 3.3)
    S = H.make_setup(nx, ny, nz, *lengths)
    ns, d = S.ns, S.decomp
    rng = np.random.default_rng(99)
    u, v, w = (rng.standard_normal((nx, ny, nz)) for _ in range(3))
    mu, rho = 0.01, 1.3

    class IC:
        Cs = 0.17
        expFilterFac = 1.5

    smag = ns.sfsmodel_smagorinsky.stress_constCs(IC(), S.geo)
    su, sv, sw = (_state(ns, d, a) for a in (u, v, w))
    mu_t = smag.eddyVisc(su, sv, sw, rho, S.metric)
    res = dict(shape=np.array([nx, ny, nz]),
               spacing=np.array([S.geo.dx, S.geo.dy, S.geo.dz]), u=u, v=v, w=w,
               mu=mu, rho=rho, Cs=IC.Cs, expFilterFac=IC.expFilterFac,
               mu_t=mu_t[2:-2, 2:-2, 2:-2].numpy().copy())
    # RHS with VISC_P = mu + mu_t (src/data/domain.py:348-352)
    VISC = torch.ones(nx + 4, ny + 4, nz + 4, dtype=torch.float64) * mu
    VISC.copy_(mu + mu_t)
    rhs = ns.velocity.rhs_NavierStokes(d, S.metric, rho, VISC, smag)
    su, sv, sw = (_state(ns, d, a) for a in (u, v, w))
    rhs.evaluate(su, sv, sw)
    res["rhs_smag"] = np.stack([rhs.rhs_u.numpy(), rhs.rhs_v.numpy(),
                                rhs.rhs_w.numpy()])
    # gradient model
    gm = ns.sfsmodel_gradient.residual_stress(d, S.geo, S.metric)
    su, sv, sw = (_state(ns, d, a) for a in (u, v, w))
    gm.update(su, sv, sw, S.metric)
    res["grad_F"] = np.stack([getattr(gm, k)[2:-2, 2:-2, 2:-2].numpy().copy()
                              for k in ("FXX", "FYY", "FZZ", "FXY", "FXZ", "FYZ")])
    VISC = torch.ones(nx + 4, ny + 4, nz + 4, dtype=torch.float64) * mu
    rhs = ns.velocity.rhs_NavierStokes(d, S.metric, rho, VISC, gm)
    su, sv, sw = (_state(ns, d, a) for a in (u, v, w))
    rhs.evaluate(su, sv, sw)
    res["rhs_grad"] = np.stack([rhs.rhs_u.numpy(), rhs.rhs_v.numpy(),
                                rhs.rhs_w.numpy()])
    np.savez_compressed(os.path.join(out, "sgs_12x16x20.npz"), **res)
    print("sgs: max mu_t", float(mu_t.abs().max()))


def adjoint_case(out):
    import torch
    nx, ny, nz = 12, 16, 20
    lengths = (2 * np.pi, 2.1, 3.3)
    S = H.make_setup(nx, ny, nz, *lengths)
    ns, d = S.ns, S.decomp
    rng = np.random.default_rng(4242)
    u, v, w = (rng.standard_normal((nx, ny, nz)) for _ in range(3))
    lu, lv, lw = (rng.standard_normal((nx, ny, nz)) for _ in range(3))
    mu, rho, dt = 0.02, 1.1, 1.0e-3

    class ZeroML:
        """'source' closure whose output is 0 * u but stays on the graph."""
        modelType = "source"

        def update(self, u_V, v_V, w_V, requires_grad=True):
            z = 0.0 * (u_V + v_V + w_V)
            self.GX = z[..., None]
            self.GY = z[..., None]
            self.GZ = z[..., None]

    VISC = torch.ones(nx + 4, ny + 4, nz + 4, dtype=torch.float64) * mu
    su, sv, sw = (_state(ns, d, a) for a in (u, v, w))
    radj = ns.adjoint.rhs_adjPredictor(d, S.metric, rho, VISC, ZeroML(), su, sv, sw)
    au, av, aw = (_state(ns, d, a) for a in (lu, lv, lw))
    radj.evaluate(au, av, aw)
    res = dict(shape=np.array([nx, ny, nz]),
               spacing=np.array([S.geo.dx, S.geo.dy, S.geo.dz]), u=u, v=v, w=w,
               lu=lu, lv=lv, lw=lw, mu=mu, rho=rho, dt=dt,
               rhs_adj=np.stack([radj.rhs_u.numpy().copy(), radj.rhs_v.numpy().copy(),
                                 radj.rhs_w.numpy().copy()]))
    # one Euler adjoint step: adjoint projection, then lam += dt rhs_adj(lam)
    au, av, aw = (_state(ns, d, a) for a in (lu, lv, lw))
    sDP = _state(ns, d, np.zeros((nx, ny, nz)))
    sp = _state(ns, d, np.zeros((nx, ny, nz)))
    src = torch.zeros(nx, ny, nz, dtype=torch.float64)
    S.metric.div_vel(au, av, aw, src)
    solver = ns.pressure.solver_bicgstab(S.comms, d, S.metric, S.geo, rho, dt,
                                         1e-13, 2000)
    solver.solve(sDP, sp, src)
    S.metric.grad_P(sDP)
    au.vel_corr(sDP.grad_x, +dt / rho)
    av.vel_corr(sDP.grad_y, +dt / rho)
    aw.vel_corr(sDP.grad_z, +dt / rho)

    class RHSSet:
        pass

    rs = RHSSet()
    rs.rhs1 = ns.adjoint.rhs_adjPredictor(d, S.metric, rho, VISC, ZeroML(), su, sv, sw)
    ns.advancer.Euler(au, av, aw, rs).step(dt)
    res["euler_adj_step"] = np.stack([au.interior().numpy().copy(),
                                      av.interior().numpy().copy(),
                                      aw.interior().numpy().copy()])
    np.savez_compressed(os.path.join(out, "adjoint_12x16x20.npz"), **res)
    print("adjoint: max |rhs_adj|", np.abs(res["rhs_adj"]).max())


def jacobi_case(out):
    import torch
    n = 16
    S = H.make_setup(n, n, n, 2 * np.pi, 2 * np.pi, 2 * np.pi)
    ns, d = S.ns, S.decomp
    rng = np.random.default_rng(77)
    src = rng.standard_normal((n, n, n))
    src -= src.mean()
    rho, dt, n_it = 1.0, 0.01, 30
    sDP = _state(ns, d, np.zeros((n, n, n)))
    sp = _state(ns, d, rng.standard_normal((n, n, n)))
    solver = ns.pressure.solver_jacobi(S.comms, d, S.metric, S.geo, rho, dt,
                                       n_it)
    srcT = torch.from_numpy(src.copy())
    r = solver.solve(sDP, sp, srcT)
    np.savez_compressed(
        os.path.join(out, "jacobi_16.npz"), shape=np.array([n, n, n]),
        spacing=np.array([S.geo.dx] * 3), source=src, rho=rho, dt=dt,
        n_it=n_it, DP=sDP.interior().numpy().copy(),
        p=sp.interior().numpy().copy(), max_res=float(r))
    print("jacobi: max_res", r)


def ml_case(out):
    """The reference's 'source' ML closure inside rhs_NavierStokes.evaluate
    (src/solver/velocity.py:360-383) with a seeded random network."""
    import torch
    n = 16
    S = H.make_setup(n, n, n, 2 * np.pi, 2 * np.pi, 2 * np.pi)
    ns, d = S.ns, S.decomp
    rng = np.random.default_rng(123)
    u, v, w = (0.5 * rng.standard_normal((n, n, n)) for _ in range(3))
    mu, rho = 0.01, 1.0

    class IC:
        simDt = 0.01

    torch.manual_seed(5)
    ml = ns.sfsmodel_ML.residual_stress(IC(), d, S.geo)
    VISC = torch.ones(n + 4, n + 4, n + 4, dtype=torch.float64) * mu
    rhs = ns.velocity.rhs_NavierStokes(d, S.metric, rho, VISC, ml)
    su, sv, sw = (_state(ns, d, a) for a in (u, v, w))
    # the closure's own inputs: the ghost-padded cell-centre interpolants
    # (the states' var_i scratch, whose last ghost layer the interpolation
    # never writes), recorded as the RHS passes them to the model
    seen = {}
    update = ml.update

    def record(a, b, c, requires_grad=False):
        seen["ci"] = np.stack([t.detach().numpy().copy() for t in (a, b, c)])
        return update(a, b, c, requires_grad)

    ml.update = record
    rhs.evaluate(su, sv, sw)
    res = dict(shape=np.array([n, n, n]), spacing=np.array([S.geo.dx] * 3), u=u, v=v,
               w=w, mu=mu, rho=rho, ci=seen["ci"],
               rhs_ml=np.stack([rhs.rhs_u.numpy(), rhs.rhs_v.numpy(), rhs.rhs_w.numpy()]))
    for k, t in ml.model.state_dict().items():
        res["w_" + k] = t.detach().numpy().copy()
    np.savez_compressed(os.path.join(out, "ml_16.npz"), **res)
    print("ml: rhs max", np.abs(res["rhs_ml"]).max())


def finalize_case(out):
    """The reference's training update (residual_stress.finalize,
    src/sfsmodel/sfsmodel_ML.py:284-349) over seven windows with seeded
    gradients: numSumDistr = 2, LR_decay = 5 (halving once epoch >= 4 and
    epoch % 5 == 0), an LR override in the configuration (which the reference
    stores but does not pass to its optimizer)."""
    import torch
    n = 8
    S = H.make_setup(n, n, n, 2 * np.pi, 2 * np.pi, 2 * np.pi)
    ns, d = S.ns, S.decomp

    class IC:
        simDt = 0.004
        modelDictSave = os.path.join(ns.tmp, "finalize_model.dict")
        LR_decay = 5
        numSumDistr = 2
        LR = 0.003

    class Comms:
        size = 1

        @staticmethod
        def parallel_sum(a):
            return a

    # every operation of the update is elementwise: the fixture keeps the
    # first K elements of every parameter (weights before and after each
    # window, the window's gradient)
    K = 96
    torch.manual_seed(11)
    ml = ns.sfsmodel_ML.residual_stress(IC(), d, S.geo)
    names = [k for k, _ in ml.model.named_parameters()]
    res = {"simDt": IC.simDt, "LR_decay": IC.LR_decay, "numSumDistr": IC.numSumDistr,
           "LR_config": IC.LR, "names": np.array(names), "K": K}
    for k, t in ml.model.named_parameters():
        res["w0_" + k] = t.detach().numpy().ravel()[:K].copy()
    rng = np.random.default_rng(77)
    epochs = 7
    for e in range(epochs):
        for k, prm in ml.model.named_parameters():
            g = (rng.standard_normal(tuple(prm.shape)) * 0.1).astype(np.float32)
            res["g%d_%s" % (e, k)] = g.ravel()[:K].copy()
            prm.grad = torch.tensor(g)
        ml.finalize(Comms())
        for k, prm in ml.model.named_parameters():
            res["w%d_%s" % (e + 1, k)] = prm.detach().numpy().ravel()[:K].copy()
        res["lr%d" % (e + 1)] = np.array([ml.LR, ml.optimizer.param_groups[0]["lr"]])
    res["epochs"] = epochs
    np.savez_compressed(os.path.join(out, "finalize_8.npz"), **res)
    print("finalize: lr", [float(res["lr%d" % (e + 1)][1]) for e in range(epochs)])


def target_case(out):
    """Domain.TargetDataVelCorr (src/data/domain.py:445-468) on a random,
    not divergence-free target field: divergence, BiCGStab solve (which also
    adds DP to the simulation pressure p), target corrected by +dt/rho grad DP."""
    import torch
    nx, ny, nz = 12, 16, 20
    lengths = (2 * np.pi, 2.1, 3.3)
    S = H.make_setup(nx, ny, nz, *lengths)
    ns, d = S.ns, S.decomp
    rng = np.random.default_rng(4321)
    uT, vT, wT = (rng.standard_normal((nx, ny, nz)) for _ in range(3))
    p0 = 0.1 * rng.standard_normal((nx, ny, nz))
    rho, dt = 1.3, 2.0e-3
    D = types.SimpleNamespace(
        targetDataVelCorr=True, metric=S.metric, rho=rho,
        state_u_T=_state(ns, d, uT), state_v_T=_state(ns, d, vT), state_w_T=_state(ns, d, wT),
        source_P=torch.zeros(nx, ny, nz, dtype=torch.float64),
        state_DP_P=_state(ns, d, np.zeros((nx, ny, nz))), state_p_P=_state(ns, d, p0),
        poisson=ns.pressure.solver_bicgstab(S.comms, d, S.metric, S.geo, rho, dt, 1e-10, 500))
    ns.domain.Domain.TargetDataVelCorr(D, dt)
    res = dict(shape=np.array([nx, ny, nz]), spacing=np.array([S.geo.dx, S.geo.dy, S.geo.dz]),
               rho=rho, dt=dt, uT=uT, vT=vT, wT=wT, p0=p0,
               u_out=D.state_u_T.interior().numpy().copy(),
               v_out=D.state_v_T.interior().numpy().copy(),
               w_out=D.state_w_T.interior().numpy().copy(),
               DP=D.state_DP_P.interior().numpy().copy(),
               p_out=D.state_p_P.interior().numpy().copy(), max_res=float(D.max_resP))
    np.savez_compressed(os.path.join(out, "target_12x16x20.npz"), **res)
    print("target: max_res", res["max_res"])


def run_case(out, n=32, steps=5, seed=0, nu=0.01, dt=0.005, stride=1):
    import torch
    ns = H.load_reference()
    import pyflow_b200.initial as ic
    u0, v0, w0 = ic.spectral_velocity((n, n, n), k0=4.0, urms=1.0, seed=seed)
    p0 = np.zeros_like(u0)
    wd = os.path.join(ns.tmp, "run_%d" % n)
    os.makedirs(wd, exist_ok=True)
    g = np.linspace(0.0, 2 * np.pi, n + 1)
    H.write_config(os.path.join(wd, "config"), g, g, g)
    H.write_restart(os.path.join(wd, "data"), [u0, v0, w0, p0], dt=dt)

    class Cfg:
        pass

    c = Cfg()
    c.configName = "restart"
    c.configFileStr = os.path.join(wd, "config")
    c.dataFileStr = os.path.join(wd, "data")
    c.dataFileType = "restart"
    c.fNameOut = os.path.join(wd, "out")
    c.numItDataOut = 1000
    c.nproc_x = c.nproc_y = c.nproc_z = 1
    c.mu, c.rho = nu, 1.0
    c.simDt, c.numIt, c.startTime = dt, steps, 0.0
    c.SFSmodel = "none"
    c.advancerName, c.equationMode = "RK4", "NS"
    c.pSolverMode = "bicgstab"
    c.min_pressure_residual, c.max_pressure_iterations = 1e-10, 1000
    c.genericOrder = 2
    c.dtypeTorch, c.dtypeNumpy = torch.float64, np.float64
    c.plotState, c.numItPlotOut = False, 20

    record = dict(dom=None, max_res=[], iters=[], stats=[])
    Dom = ns.domain.Domain
    orig_fs = Dom.forwardStep
    orig_apply = ns.pressure.Pressure_Base.applyOperator
    count = [0]

    def apply_counting(self, A, B):
        count[0] += 1
        return orig_apply(self, A, B)

    def fs(self, simDt):
        record["dom"] = self
        count[0] = 0
        orig_fs(self, simDt)
        record["max_res"].append(float(self.max_resP))
        record["iters"].append(count[0] // 2)
        u = self.state_u_P.interior()
        v = self.state_v_P.interior()
        w = self.state_w_P.interior()
        st = [float(torch.max(torch.abs(a))) for a in (u, v, w)]
        tke = float(torch.sum(u ** 2 + v ** 2 + w ** 2)) / float(n ** 3) * 0.5
        dv = torch.zeros(n, n, n, dtype=torch.float64)
        self.metric.div_vel(self.state_u_P, self.state_v_P, self.state_w_P, dv)
        record["stats"].append(st + [tke, float(torch.max(torch.abs(dv)))])

    Dom.forwardStep = fs
    ns.pressure.Pressure_Base.applyOperator = apply_counting
    os.environ["PF_FAKE_RANK"] = "1"  # skip rank-0 monitor/restart file output
    try:
        ns.PyFlow.run(c)
    finally:
        Dom.forwardStep = orig_fs
        ns.pressure.Pressure_Base.applyOperator = orig_apply
        os.environ.pop("PF_FAKE_RANK", None)
    D = record["dom"]
    if stride > 1:
        # large case: the initial field is regenerated from its seed by the
        # tests; keep the final fields on a strided subset plus their moments
        fields = {k: getattr(D, "state_%s_P" % k).interior().numpy().copy()
                  for k in ("u", "v", "w", "p")}
        sub = {k + "_sub": a[::stride, ::stride, ::stride].copy() for k, a in fields.items()}
        mom = np.array([[a.sum(), (a * a).sum(), np.abs(a).max()] for a in fields.values()])
        np.savez_compressed(
            os.path.join(out, "run_%d.npz" % n), shape=np.array([n, n, n]),
            spacing=np.array([2 * np.pi / n] * 3), seed=seed, k0=4.0, urms=1.0, nu=nu,
            rho=1.0, dt=dt, steps=steps, stride=stride, moments=mom,
            max_res=np.array(record["max_res"]), iters=np.array(record["iters"]),
            stats=np.array(record["stats"]), **sub)
        print("run %d: iters" % n, record["iters"], "max_res", record["max_res"])
        return
    np.savez_compressed(
        os.path.join(out, "run_%d.npz" % n), shape=np.array([n, n, n]),
        spacing=np.array([2 * np.pi / n] * 3), seed=seed, nu=nu, rho=1.0,
        dt=dt, steps=steps, u0=u0, v0=v0, w0=w0,
        u=D.state_u_P.interior().numpy().copy(),
        v=D.state_v_P.interior().numpy().copy(),
        w=D.state_w_P.interior().numpy().copy(),
        p=D.state_p_P.interior().numpy().copy(),
        max_res=np.array(record["max_res"]), iters=np.array(record["iters"]),
        stats=np.array(record["stats"]))
    print("run: iters", record["iters"], "max_res", record["max_res"])


if __name__ == "__main__":
    out = HERE
    which = sys.argv[1:] or ["ops", "jacobi", "sgs", "adjoint", "run", "run64", "ml",
                             "finalize", "target"]
    if "ops" in which:
        ops_case(out)
    if "jacobi" in which:
        jacobi_case(out)
    if "sgs" in which:
        sgs_case(out)
    if "adjoint" in which:
        adjoint_case(out)
    if "run" in which:
        run_case(out)
    if "ml" in which:
        ml_case(out)
    if "finalize" in which:
        finalize_case(out)
    if "target" in which:
        target_case(out)
    if "run64" in which:
        # the 64^3 plain-DNS workload: seed 0, k0 = 4, nu = 0.01, dt = 0.005,
        # 20 RK4 steps, BiCGStab to 1e-10
        run_case(out, n=64, steps=20, stride=4)
