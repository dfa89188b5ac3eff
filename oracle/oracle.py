"""ctypes wrapper of the CPU oracle ``liboracle.so`` (built from pf_oracle.c).

TEST INFRASTRUCTURE ONLY.  Only tests/, ``__graft_entry__.smoke()`` and
bench.py's CPU-baseline / reference arm import this module, always as the
checker or the timed CPU baseline, never as part of the product path.

All arrays are C-contiguous float64 numpy arrays of shape (nx, ny, nz), the
ghost-free interior of the reference's ``state_P.var`` (src/data/state.py:142-146).
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None


class Grid(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
                ("dx", ctypes.c_double), ("dy", ctypes.c_double),
                ("dz", ctypes.c_double)]


def build():
    """Compile liboracle.so with the committed Makefile."""
    import subprocess
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        P = ctypes.c_void_p
        D = ctypes.c_double
        I = ctypes.c_int
        G = ctypes.POINTER(Grid)
        L.or_rhs_ns.argtypes = [G, P, P, P, P, D, D, P, P, P, P]
        L.or_rk4_step.argtypes = [G, P, P, P, P, D, D, P, D]
        L.or_euler_step.argtypes = [G, P, P, P, P, D, D, P, D]
        L.or_div_vel.argtypes = [G, P, P, P, P]
        L.or_laplace_apply.argtypes = [G, P, P]
        L.or_bicgstab.argtypes = [G, D, D, D, I, P, P, P,
                                  ctypes.POINTER(I), ctypes.POINTER(I)]
        L.or_bicgstab.restype = D
        L.or_jacobi.argtypes = [G, D, D, I, P, P, P]
        L.or_jacobi.restype = D
        L.or_vel_corr.argtypes = [G, P, D, P, P, P]
        L.or_forward_step.argtypes = [G, P, P, P, P, P, P, D, D, P, D, I, I, D,
                                      I, ctypes.POINTER(I)]
        L.or_forward_step.restype = D
        L.or_stats.argtypes = [G, P, P, P, P]
        _lib = L
    return _lib


def grid(shape, spacing):
    return Grid(int(shape[0]), int(shape[1]), int(shape[2]),
                float(spacing[0]), float(spacing[1]), float(spacing[2]))


def _p(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def rhs_ns(spacing, u, v, w, mu, rho, visc=None, sfs=None):
    """rhs_NavierStokes.evaluate (src/solver/velocity.py:221-355)."""
    u, v, w = _f64(u), _f64(v), _f64(w)
    g = grid(u.shape, spacing)
    out = [np.empty_like(u) for _ in range(3)]
    visc = None if visc is None else _f64(visc)
    sfs = None if sfs is None else _f64(np.stack(sfs))
    lib().or_rhs_ns(ctypes.byref(g), _p(u), _p(v), _p(w), _p(visc), mu, rho,
                    _p(sfs), _p(out[0]), _p(out[1]), _p(out[2]))
    return out


def rk4_step(spacing, u, v, w, mu, rho, dt, visc=None, sfs=None):
    """RK4.step predictor (src/solver/advancer.py:75-113); returns new u,v,w."""
    u, v, w = _f64(u).copy(), _f64(v).copy(), _f64(w).copy()
    g = grid(u.shape, spacing)
    visc = None if visc is None else _f64(visc)
    sfs = None if sfs is None else _f64(np.stack(sfs))
    lib().or_rk4_step(ctypes.byref(g), _p(u), _p(v), _p(w), _p(visc), mu, rho,
                      _p(sfs), dt)
    return u, v, w


def div_vel(spacing, u, v, w):
    """metric_uniform.div_vel (src/metric/metric_staggered.py:438-453)."""
    u, v, w = _f64(u), _f64(v), _f64(w)
    g = grid(u.shape, spacing)
    d = np.empty_like(u)
    lib().or_div_vel(ctypes.byref(g), _p(u), _p(v), _p(w), _p(d))
    return d


def laplace_apply(spacing, a):
    """Pressure_Base.applyOperator (src/solver/pressure.py:54-84)."""
    a = _f64(a)
    g = grid(a.shape, spacing)
    b = np.empty_like(a)
    lib().or_laplace_apply(ctypes.byref(g), _p(a), _p(b))
    return b


def bicgstab(spacing, source, p, rho, dt, min_res, max_it):
    """solver_bicgstab.solve (src/solver/pressure.py:196-297).

    Returns (DP, p_new, max_res, iterations, status)."""
    src = _f64(source).copy()
    p = _f64(p).copy()
    g = grid(src.shape, spacing)
    DP = np.zeros_like(src)
    it = ctypes.c_int(0)
    st = ctypes.c_int(0)
    r = lib().or_bicgstab(ctypes.byref(g), rho, dt, min_res, int(max_it),
                          _p(DP), _p(p), _p(src), ctypes.byref(it),
                          ctypes.byref(st))
    return DP, p, r, it.value, st.value


def jacobi(spacing, source, rho, dt, n_it):
    """solver_jacobi.solve (src/solver/pressure.py:115-161).

    Returns (DP = iterate n-1, p = iterate n, max_res)."""
    src = _f64(source).copy()
    g = grid(src.shape, spacing)
    p = np.zeros_like(src)
    DP = np.zeros_like(src)
    r = lib().or_jacobi(ctypes.byref(g), rho, dt, int(n_it), _p(DP), _p(p),
                        _p(src))
    return DP, p, r


def vel_corr(spacing, DP, scale, u, v, w):
    """grad_P + vel_corr (metric_staggered.py:390-401, state.py:198-211)."""
    u, v, w = _f64(u).copy(), _f64(v).copy(), _f64(w).copy()
    DP = _f64(DP)
    g = grid(u.shape, spacing)
    lib().or_vel_corr(ctypes.byref(g), _p(DP), scale, _p(u), _p(v), _p(w))
    return u, v, w


def forward_step(spacing, u, v, w, p, mu, rho, dt, visc=None, sfs=None,
                 rk4=True, solver="bicgstab", min_res=1e-10, max_it=300):
    """Domain.forwardStep (src/data/domain.py:342-402) with SFS off or tensor.

    Returns (u, v, w, p, DP, max_res, iterations)."""
    u, v, w, p = (_f64(a).copy() for a in (u, v, w, p))
    g = grid(u.shape, spacing)
    DP = np.zeros_like(u)
    visc = None if visc is None else _f64(visc)
    sfs = None if sfs is None else _f64(np.stack(sfs))
    it = ctypes.c_int(0)
    r = lib().or_forward_step(ctypes.byref(g), _p(u), _p(v), _p(w), _p(p),
                              _p(DP), _p(visc), mu, rho, _p(sfs), dt,
                              1 if rk4 else 0,
                              0 if solver == "bicgstab" else 1, min_res,
                              int(max_it), ctypes.byref(it))
    return u, v, w, p, DP, r, it.value


def stats(spacing, u, v, w):
    """Per-step monitor statistics (src/core/PyFlow.py:379-395):
    (max|u|, max|v|, max|w|, TKE, max|div u|)."""
    u, v, w = _f64(u), _f64(v), _f64(w)
    g = grid(u.shape, spacing)
    out = np.zeros(5)
    lib().or_stats(ctypes.byref(g), _p(u), _p(v), _p(w), _p(out))
    return out


def grad_center(spacing, u, v, w):
    """Cell-centred velocity gradients of metric_uniform.grad_vel_center
    (src/metric/metric_staggered.py:215-268) with periodic wrap, as numpy:
    the normal derivative is the difference of the two face values, a
    transverse derivative the difference of the face-to-centre interpolant
    averaged back to the neighbouring faces.  Returns the nine arrays
    (ux, uy, uz, vx, vy, vz, wx, wy, wz)."""
    u, v, w = _f64(u), _f64(v), _f64(w)
    dxi, dyi, dzi = (1.0 / s for s in spacing)
    sh = lambda a, ax, k: np.roll(a, -k, axis=ax)   # a[i + k] along ax

    def tangential(f, ax_c, ax_t, di):
        c0 = 0.5 * (sh(f, ax_c, 1) + f)          # value at the cell centre
        cp, cm = sh(c0, ax_t, 1), sh(c0, ax_t, -1)
        return (0.5 * (cp + c0) - 0.5 * (c0 + cm)) * di

    ux = (sh(u, 0, 1) - u) * dxi
    vy = (sh(v, 1, 1) - v) * dyi
    wz = (sh(w, 2, 1) - w) * dzi
    return (ux, tangential(u, 0, 1, dyi), tangential(u, 0, 2, dzi),
            tangential(v, 1, 0, dxi), vy, tangential(v, 1, 2, dzi),
            tangential(w, 2, 0, dxi), tangential(w, 2, 1, dyi), wz)


def flow_stats(spacing, u, v, w, nu):
    """Monitor statistics (src/core/PyFlow.py:379-395) plus the dissipation
    rate eps = 2 nu <S_ij S_ij> of the cell-centred strain rate built from
    grad_center: (max|u|, max|v|, max|w|, TKE, max|div u|, eps)."""
    st = stats(spacing, u, v, w)
    ux, uy, uz, vx, vy, vz, wx, wy, wz = grad_center(spacing, u, v, w)
    s12, s13, s23 = 0.5 * (uy + vx), 0.5 * (uz + wx), 0.5 * (vz + wy)
    ss = ((ux * ux + vy * vy) + wz * wz) + 2.0 * ((s12 * s12 + s13 * s13) + s23 * s23)
    return np.concatenate([st, [2.0 * nu * ss.mean()]])
