"""Operator-level entry points on torch CUDA tensors.

Each function validates its tensors (CUDA, contiguous, dtype), owns no device
memory beyond a cached workspace tensor per device, and calls one C-ABI entry
point of libpyflow_b200.so on torch's current stream.  Fields are ghost-free
(nx, ny, nz) tensors, z contiguous -- the interior of the reference's
``state_P.var`` (src/data/state.py:142-146).
"""
import ctypes

import torch

from . import _lib as L

PREC = {"fp64": L.PF_FP64, "mixed": L.PF_MIXED, "mixed_mg": L.PF_MIXED_MG}
_ws_cache = {}


def grid(shape, spacing):
    nx, ny, nz = (int(s) for s in shape)
    dx, dy, dz = (float(h) for h in spacing)
    return L.Grid(nx, ny, nz, dx, dy, dz)


def _p(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def _check(t, shape, dtype, name):
    if not isinstance(t, torch.Tensor):
        raise TypeError("%s must be a torch tensor" % name)
    if not t.is_cuda:
        raise ValueError("%s must be a CUDA tensor (there is no CPU path)" % name)
    if not t.is_contiguous():
        raise ValueError("%s must be contiguous" % name)
    if t.dtype != dtype:
        raise TypeError("%s must be %s, got %s" % (name, dtype, t.dtype))
    if tuple(t.shape) != tuple(shape):
        raise ValueError("%s has shape %s, expected %s" % (name, tuple(t.shape), tuple(shape)))


def _stream(t):
    return ctypes.c_void_p(torch.cuda.current_stream(t.device).cuda_stream)


def workspace(g, prec, device):
    """A cached uint8 workspace of at least pf_workspace_bytes(g, prec)."""
    need = L.lib().pf_workspace_bytes(ctypes.byref(g), prec)
    if need == 0:
        raise ValueError("invalid grid or precision")
    key = torch.device(device)
    ws = _ws_cache.get(key)
    if ws is None or ws.numel() < need:
        _ws_cache[key] = None
        ws = torch.empty(need, dtype=torch.uint8, device=key)
        _ws_cache[key] = ws
    return ws


def rhs_ns(u, v, w, spacing, mu, rho, visc=None, sfs=None, out=None):
    """rhs_NavierStokes.evaluate (src/solver/velocity.py:221-355).

    dtype float64 computes in FP64 (reference order), float32 in FP32."""
    dt = u.dtype
    prec = L.PF_FP64 if dt == torch.float64 else L.PF_MIXED
    for t, nm in ((u, "u"), (v, "v"), (w, "w")):
        _check(t, u.shape, dt, nm)
    if visc is not None:
        _check(visc, u.shape, dt, "visc")
    if sfs is not None:
        _check(sfs, (6,) + tuple(u.shape), dt, "sfs")
    if out is None:
        out = tuple(torch.empty_like(u) for _ in range(3))
    g = grid(u.shape, spacing)
    L.check("pf_rhs_ns", L.lib().pf_rhs_ns(
        ctypes.byref(g), prec, _p(u), _p(v), _p(w), _p(visc), float(mu),
        float(rho), _p(sfs), _p(out[0]), _p(out[1]), _p(out[2]), _stream(u)))
    return out


def div_vel(u, v, w, spacing, out=None):
    """metric_uniform.div_vel (src/metric/metric_staggered.py:438-453)."""
    for t, nm in ((u, "u"), (v, "v"), (w, "w")):
        _check(t, u.shape, torch.float64, nm)
    out = torch.empty_like(u) if out is None else out
    g = grid(u.shape, spacing)
    L.check("pf_div_vel", L.lib().pf_div_vel(
        ctypes.byref(g), _p(u), _p(v), _p(w), _p(out), _stream(u)))
    return out


def laplace_apply(A, spacing, out=None):
    """Pressure_Base.applyOperator (src/solver/pressure.py:54-84)."""
    _check(A, A.shape, torch.float64, "A")
    out = torch.empty_like(A) if out is None else out
    g = grid(A.shape, spacing)
    L.check("pf_laplace_apply", L.lib().pf_laplace_apply(
        ctypes.byref(g), _p(A), _p(out), _stream(A)))
    return out


def predictor_step(u, v, w, spacing, mu, rho, dt, rk4=True, prec="fp64",
                   visc=None, sfs=None):
    """RK4.step / Euler.step (src/solver/advancer.py:41-113); in place."""
    pr = PREC[prec]
    for t, nm in ((u, "u"), (v, "v"), (w, "w")):
        _check(t, u.shape, torch.float64, nm)
    sdt = torch.float64 if pr == L.PF_FP64 else torch.float32
    if visc is not None:
        _check(visc, u.shape, sdt, "visc")
    if sfs is not None:
        _check(sfs, (6,) + tuple(u.shape), sdt, "sfs")
    g = grid(u.shape, spacing)
    ws = workspace(g, pr, u.device)
    L.check("pf_predictor_step", L.lib().pf_predictor_step(
        ctypes.byref(g), pr, 1 if rk4 else 0, _p(u), _p(v), _p(w), _p(visc),
        float(mu), float(rho), _p(sfs), float(dt), _p(ws), ws.numel(),
        _stream(u)))


def bicgstab_solve(source, DP, p, spacing, rho, dt, min_res, max_it,
                   prec="fp64", warm=False):
    """solver_bicgstab.solve (src/solver/pressure.py:196-297): DP solves the
    pressure Poisson equation for the divergence ``source``; p += DP.  With
    ``warm`` (mixed forms) the solve starts from the DP given.
    Returns a SolveInfo (max_res, iterations, outer, status)."""
    for t, nm in ((source, "source"), (DP, "DP"), (p, "p")):
        _check(t, source.shape, torch.float64, nm)
    pr = PREC[prec]
    flag = L.PF_WARM_START if warm else 0
    g = grid(source.shape, spacing)
    ws = workspace(g, pr, source.device)
    info = L.SolveInfo()
    L.check("pf_bicgstab_solve", L.lib().pf_bicgstab_solve(
        ctypes.byref(g), pr | flag, float(rho), float(dt), float(min_res),
        int(max_it), _p(source), _p(DP), _p(p), _p(ws), ws.numel(),
        _stream(source), ctypes.byref(info)))
    return info


def jacobi_solve(source, pold, p, spacing, rho, dt, n_it):
    """solver_jacobi.solve (src/solver/pressure.py:115-161). Returns max_res."""
    for t, nm in ((source, "source"), (pold, "pold"), (p, "p")):
        _check(t, source.shape, torch.float64, nm)
    g = grid(source.shape, spacing)
    ws = workspace(g, L.PF_FP64, source.device)
    r = ctypes.c_double(0.0)
    L.check("pf_jacobi_solve", L.lib().pf_jacobi_solve(
        ctypes.byref(g), float(rho), float(dt), int(n_it), _p(source),
        _p(pold), _p(p), _p(ws), ws.numel(), _stream(source), ctypes.byref(r)))
    return r.value


def vel_corr(DP, scale, u, v, w, spacing):
    """grad_P + vel_corr (src/metric/metric_staggered.py:390-401,
    src/data/state.py:198-211)."""
    for t, nm in ((DP, "DP"), (u, "u"), (v, "v"), (w, "w")):
        _check(t, DP.shape, torch.float64, nm)
    g = grid(DP.shape, spacing)
    L.check("pf_vel_corr", L.lib().pf_vel_corr(
        ctypes.byref(g), _p(DP), float(scale), _p(u), _p(v), _p(w),
        _stream(DP)))


def forward_step(u, v, w, p, DP, spacing, mu, rho, dt, rk4=True,
                 solver="bicgstab", min_res=1e-10, max_it=300, prec="fp64",
                 visc=None, sfs=None, warm=False):
    """Domain.forwardStep + velCorr (src/data/domain.py:342-402).  With
    ``warm`` (mixed forms) the pressure solve starts from the DP given (the
    previous step's), as the mixed step plans do."""
    for t, nm in ((u, "u"), (v, "v"), (w, "w"), (p, "p"), (DP, "DP")):
        _check(t, u.shape, torch.float64, nm)
    pr = PREC[prec]
    sdt = torch.float64 if pr == L.PF_FP64 else torch.float32
    if visc is not None:
        _check(visc, u.shape, sdt, "visc")
    if sfs is not None:
        _check(sfs, (6,) + tuple(u.shape), sdt, "sfs")
    g = grid(u.shape, spacing)
    ws = workspace(g, pr, u.device)
    info = L.SolveInfo()
    L.check("pf_forward_step", L.lib().pf_forward_step(
        ctypes.byref(g), pr | (L.PF_WARM_START if warm else 0), 1 if rk4 else 0,
        0 if solver == "bicgstab" else 1, _p(u), _p(v), _p(w), _p(p), _p(DP),
        _p(visc), float(mu), float(rho), _p(sfs), float(dt), float(min_res),
        int(max_it), _p(ws), ws.numel(), _stream(u), ctypes.byref(info)))
    return info


def stats(u, v, w, spacing, out=None):
    """Monitor statistics (src/core/PyFlow.py:379-395) as a device tensor
    [max|u|, max|v|, max|w|, TKE, max|div u|]."""
    for t, nm in ((u, "u"), (v, "v"), (w, "w")):
        _check(t, u.shape, torch.float64, nm)
    out = torch.empty(5, dtype=torch.float64, device=u.device) if out is None else out
    g = grid(u.shape, spacing)
    ws = workspace(g, L.PF_FP64, u.device)
    L.check("pf_stats", L.lib().pf_stats(
        ctypes.byref(g), _p(u), _p(v), _p(w), _p(out), _p(ws), ws.numel(),
        _stream(u)))
    return out


def flow_stats(u, v, w, spacing, nu, out=None):
    """Monitor statistics plus the dissipation rate (pf_flow_stats) as a
    device tensor [max|u|, max|v|, max|w|, TKE, max|div u|, eps], with
    eps = 2 nu <S_ij S_ij> from the cell-centred strain rate of
    metric_uniform.grad_vel_center (src/metric/metric_staggered.py:215-268)."""
    for t, nm in ((u, "u"), (v, "v"), (w, "w")):
        _check(t, u.shape, torch.float64, nm)
    out = torch.empty(6, dtype=torch.float64, device=u.device) if out is None else out
    g = grid(u.shape, spacing)
    ws = workspace(g, L.PF_FP64, u.device)
    L.check("pf_flow_stats", L.lib().pf_flow_stats(
        ctypes.byref(g), _p(u), _p(v), _p(w), float(nu), _p(out), _p(ws), ws.numel(),
        _stream(u)))
    return out


SGS_MODELS = {"smagorinsky": (0, 1), "gradient": (1, 6), "gradients": (2, 9)}


def sgs_closure(model, u, v, w, spacing, coef=1.0, out=None):
    """Cell-centred SGS closure fields (pf_sgs_closure): 'smagorinsky' ->
    (nx,ny,nz) eddy viscosity coef*|S|; 'gradient' -> (6,nx,ny,nz) stresses
    coef du_i/dx_k du_j/dx_k; 'gradients' -> (9,nx,ny,nz) velocity gradients."""
    mid, nf = SGS_MODELS[model]
    for t, nm in ((u, "u"), (v, "v"), (w, "w")):
        _check(t, u.shape, torch.float64, nm)
    shape = tuple(u.shape) if nf == 1 else (nf,) + tuple(u.shape)
    if out is None or tuple(out.shape) != shape:
        out = torch.empty(shape, dtype=torch.float64, device=u.device)
    g = grid(u.shape, spacing)
    L.check("pf_sgs_closure", L.lib().pf_sgs_closure(
        ctypes.byref(g), mid, _p(u), _p(v), _p(w), float(coef), _p(out),
        _stream(u)))
    return out


def mlsrc_pack(params, norm, pack=None):
    """Pack the 'source' network for pf_mlsrc_closure (pf_mlsrc_pack).

    params: the 12 float32 CUDA tensors fc1.weight, fc1.bias, fcG.weight,
    fcG.bias, fcG2.weight, fcG2.bias, fc2.weight, fc2.bias, fc3.weight,
    fc3.bias, fc4.weight, fc4.bias; norm: the 21 feature normalisation
    constants (float32, CUDA)."""
    ts = [t.detach().contiguous() for t in list(params) + [norm]]
    if len(ts) != 13:
        raise ValueError("expected 12 parameter tensors and the normalisation")
    for i, t in enumerate(ts):
        if not t.is_cuda or t.dtype != torch.float32:
            raise TypeError("parameter %d must be a float32 CUDA tensor" % i)
    nbytes = L.lib().pf_mlsrc_pack_bytes()
    if pack is None or pack.numel() < nbytes:
        pack = torch.empty(nbytes, dtype=torch.uint8, device=ts[0].device)
    arr = (ctypes.c_void_p * 13)(*[t.data_ptr() for t in ts])
    L.check("pf_mlsrc_pack", L.lib().pf_mlsrc_pack(arr, _p(pack), _stream(ts[0])))
    return pack


def mlsrc_closure(u, v, w, dx, pack, G=None, S=None, err=None):
    """The 'source' closure (pf_mlsrc_closure): returns (G, S, err), G the
    (3, nx, ny, nz) FP64 closure terms GX, GY, GZ at cell centres, S the face
    sources the RHS subtracts, err a device int (1 if a tensor-core wait
    timed out)."""
    for t, nm in ((u, "u"), (v, "v"), (w, "w")):
        _check(t, u.shape, torch.float64, nm)
    shape = (3,) + tuple(u.shape)
    if G is None:
        G = torch.empty(shape, dtype=torch.float64, device=u.device)
    if S is None:
        S = torch.empty(shape, dtype=torch.float64, device=u.device)
    if err is None:
        err = torch.zeros(1, dtype=torch.int32, device=u.device)
    g = grid(u.shape, (dx, dx, dx))
    need = L.lib().pf_mlsrc_workspace_bytes(ctypes.byref(g))
    key = ("mlsrc", torch.device(u.device))
    ws = _ws_cache.get(key)
    if ws is None or ws.numel() < need:
        _ws_cache[key] = None
        ws = torch.empty(need, dtype=torch.uint8, device=u.device)
        _ws_cache[key] = ws
    L.check("pf_mlsrc_closure", L.lib().pf_mlsrc_closure(
        ctypes.byref(g), _p(u), _p(v), _p(w), _p(pack), _p(G), _p(S), _p(ws),
        ctypes.c_size_t(ws.numel()), _p(err), _stream(u)))
    return G, S, err
