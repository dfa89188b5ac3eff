"""The hand-written adjoint (pf_rhs_adjoint, pf_sfs_adjoint,
pyflow_b200.adjoint) against the reference's own adjoint and finite
differences.

* The reference's adjoint RHS (rhs_adjPredictor.evaluate) is the exact
  transpose of its forward Jacobian (a dot-product test against the oracle
  agrees to 1e-16), so pf_rhs_adjoint must reproduce it to round-off.
* One Euler adjoint step (adjoint projection + adjoint advancer) must match
  the reference's Euler adjoint step to the Poisson tolerance.
* The stage-exact RK4 adjoint of a multi-step window must match central
  finite differences of the objective to 1e-5 (the BiCGStab tolerance is
  1e-13 in these checks so the forward map is smooth at the FD scale).
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def cu(a):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")


@pytest.fixture(scope="module")
def A():
    import pyflow_b200.adjoint as A
    return A


def test_rhs_adjoint_matches_reference(A, golden):
    g = golden("adjoint_12x16x20.npz")
    out = A.rhs_adjoint((cu(g["u"]), cu(g["v"]), cu(g["w"])),
                        (cu(g["lu"]), cu(g["lv"]), cu(g["lw"])), g["spacing"],
                        float(g["mu"]), float(g["rho"]))
    got = np.stack([t.cpu().numpy() for t in out])
    ref = g["rhs_adj"]
    assert np.abs(got - ref).max() <= 1e-13 * np.abs(ref).max()


def test_rhs_adjoint_dot_product(A):
    """<J(u) v, lam> == <v, J(u)^T lam>; J v is exact by central differences
    because the RHS is quadratic in the velocity."""
    import pyflow_b200.ops as ops
    rng = np.random.default_rng(3)
    shape, sp = (40, 33, 48), (0.11, 0.07, 0.09)
    u, v, w, lu, lv, lw, du, dv, dw = (cu(rng.standard_normal(shape)) for _ in range(9))
    fp = ops.rhs_ns(u + du, v + dv, w + dw, sp, 0.013, 1.2)
    fm = ops.rhs_ns(u - du, v - dv, w - dw, sp, 0.013, 1.2)
    lhs = sum(float(((a - b) * 0.5 * l).sum()) for a, b, l in zip(fp, fm, (lu, lv, lw)))
    at = A.rhs_adjoint((u, v, w), (lu, lv, lw), sp, 0.013, 1.2)
    rhs = sum(float((d * a).sum()) for d, a in zip((du, dv, dw), at))
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)


def test_euler_adjoint_step_matches_reference(A, golden):
    g = golden("adjoint_12x16x20.npz")
    lam, _ = A.step_vjp((cu(g["u"]), cu(g["v"]), cu(g["w"])),
                        (cu(g["lu"]), cu(g["lv"]), cu(g["lw"])), g["spacing"],
                        float(g["mu"]), float(g["rho"]), float(g["dt"]), rk4=False,
                        tol=1e-13)
    got = np.stack([t.cpu().numpy() for t in lam])
    ref = g["euler_adj_step"]
    assert np.abs(got - ref).max() <= 1e-9 * np.abs(ref).max()


def _window(A, u0, sp, mu, dt, steps, sfs=None):
    u, v, w = u0
    for _ in range(steps):
        u, v, w = A.forward_step(u, v, w, sp, mu, 1.0, dt, sfs=sfs, tol=1e-13)
    return 0.5 * ((u * u).sum() + (v * v).sum() + (w * w).sum())


@pytest.mark.parametrize("rk4", [True, False])
def test_window_gradient_vs_finite_differences(A, rk4):
    import pyflow_b200.initial as ic
    n = 16
    sp = (2 * np.pi / n,) * 3
    mu, dt, steps = 0.05, 0.01, 3
    base = [cu(a) for a in ic.spectral_velocity((n, n, n), k0=2.0, seed=11)]
    x = [t.clone().requires_grad_(True) for t in base]
    u, v, w = x
    for _ in range(steps):
        u, v, w = A.forward_step(u, v, w, sp, mu, 1.0, dt, rk4=rk4, tol=1e-13)
    L = 0.5 * ((u * u).sum() + (v * v).sum() + (w * w).sum())
    L.backward()
    grad = [t.grad for t in x]
    rng = np.random.default_rng(8)
    delta = [cu(rng.standard_normal((n, n, n))) for _ in range(3)]
    eps = 1e-4

    def Lof(s):
        uu, vv, ww = (b + s * d for b, d in zip(base, delta))
        with torch.no_grad():
            for _ in range(steps):
                uu, vv, ww = A.forward_step(uu, vv, ww, sp, mu, 1.0, dt, rk4=rk4, tol=1e-13)
            return float(0.5 * ((uu * uu).sum() + (vv * vv).sum() + (ww * ww).sum()))

    fd = (Lof(eps) - Lof(-eps)) / (2 * eps)
    ad = sum(float((g_ * d).sum()) for g_, d in zip(grad, delta))
    assert abs(fd - ad) <= 1e-5 * abs(ad), (fd, ad)


def test_sfs_stress_gradient_vs_finite_differences(A):
    """dL/dF for 'tensor' SFS stresses held fixed over an RK4 step."""
    import pyflow_b200.initial as ic
    n = 16
    sp = (2 * np.pi / n,) * 3
    u0 = [cu(a) for a in ic.spectral_velocity((n, n, n), k0=2.0, seed=12)]
    rng = np.random.default_rng(9)
    F = cu(0.05 * rng.standard_normal((6, n, n, n))).requires_grad_(True)
    u, v, w = A.forward_step(*u0, sp, 0.02, 1.0, 0.01, sfs=F, tol=1e-13)
    L = 0.5 * ((u * u).sum() + (v * v).sum() + (w * w).sum())
    L.backward()
    dF = cu(rng.standard_normal((6, n, n, n)))
    eps = 1e-4

    def Lof(s):
        with torch.no_grad():
            uu, vv, ww = A.forward_step(*u0, sp, 0.02, 1.0, 0.01,
                                        sfs=(F.detach() + s * dF).contiguous(), tol=1e-13)
            return float(0.5 * ((uu * uu).sum() + (vv * vv).sum() + (ww * ww).sum()))

    fd = (Lof(eps) - Lof(-eps)) / (2 * eps)
    ad = float((F.grad * dF).sum())
    assert abs(fd - ad) <= 1e-5 * abs(ad), (fd, ad)
