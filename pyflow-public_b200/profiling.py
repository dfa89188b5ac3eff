"""Per-kernel device timing and the HBM roofline byte model.

``enable(True)`` makes the library bracket each of its kernel launches with
CUDA events on the launching stream; ``read()`` returns {kernel: {launches,
ms}}.  ``roofline()`` turns those times into achieved GB/s with the
algorithmic (compulsory) bytes each kernel must move per launch: every field
it reads or writes counted once per cell, stencil neighbours not recounted.
"""
import ctypes
import json
import os

from . import _lib as L


class _KT(ctypes.Structure):
    _fields_ = [("name", ctypes.c_char * 48), ("launches", ctypes.c_longlong),
                ("ms", ctypes.c_double)]


_lib = L.lib()
_lib.pf_profile_enable.argtypes = [ctypes.c_int]
_lib.pf_profile_enable.restype = ctypes.c_int
_lib.pf_profile_read.argtypes = [ctypes.POINTER(_KT), ctypes.c_int,
                                 ctypes.POINTER(ctypes.c_int)]
_lib.pf_profile_read.restype = ctypes.c_int


def enable(on=True):
    _lib.pf_profile_enable(1 if on else 0)


def read():
    cnt = ctypes.c_int(0)
    _lib.pf_profile_read(None, 0, ctypes.byref(cnt))
    arr = (_KT * max(1, cnt.value))()
    _lib.pf_profile_read(arr, cnt.value, ctypes.byref(cnt))
    return {arr[i].name.decode(): {"launches": int(arr[i].launches),
                                   "ms": float(arr[i].ms)}
            for i in range(cnt.value)}


def bytes_per_cell(name):
    """Algorithmic bytes per cell of one launch of ``name``."""
    f64 = name.endswith("_f64")
    s = 8 if f64 else 4
    table = {
        # BiCGStab: kernel CA reads res, pp, vv, t, x, res0 and writes x,
        # res', pp', vv'; kernel B reads res', vv', res0 and writes t
        # -> 14 field passes per iteration
        "bicg_ca": 10 * s, "bicg_b": 4 * s,
        # init: read source (f64), write res, res0, x, pp, vv, t
        "bicg_init": 8 + 6 * s,
        # RK4 stages: FP64 state u,v,w (24 B) + stage state / k-sum (3 fields)
        "rhs_first": 24 + 6 * s, "rhs_mid": 24 + 12 * s,
        "rhs_last": 24 + 6 * s + 24, "rhs_euler": 48, "rhs_rhs": 6 * s,
    }
    for k, v in table.items():
        if name.startswith(k):
            return v
    fixed = {
        # multigrid-preconditioned FP32 BiCGStab (finest-level launches only;
        # coarse levels have their own names and fewer cells)
        "mg_smooth0_p": 20, "mg_smooth0_s": 16, "mg_smooth_l0": 12,
        "mg_restrict_l0": 8.5, "mg_prolong_l0": 8.5, "mg_av": 12, "mg_at": 12,
        "mg_update": 32, "mg_init": 16, "fold_correction": 20,
        # warm-started mixed solves: source in, b out (a cold start also
        # clears DP: 24)
        "mixed_b_init": 16, "mixed_update": 20, "mixed_residual": 24,
        "add_inplace": 24, "div_vel": 32, "vel_corr": 56, "stats": 24,
        "laplace_apply": 16, "jacobi_sweep": 24, "jacobi_prep": 24,
        "jacobi_residual": 16,
        # x-slab BiCGStab (FP64, per interior cell): 21 field passes per
        # iteration in the reference's order of operations
        "slab_pupdate": 32, "slab_apply_p": 24, "slab_supdate": 48,
        "slab_apply_s": 16, "slab_final": 48, "slab_init": 64, "slab_add": 24}
    return fixed.get(name)


def peaks():
    """Measured HBM bandwidth (GB/s) of this pool's B200s, with its source."""
    here = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    path = os.path.join(here, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            pk = json.load(f)
        return float(pk["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def tensor_peak():
    """Measured dense BF16 tensor throughput (TFLOP/s, the burst figure for a
    kernel timed alone) with its source."""
    here = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    path = os.path.join(here, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            pk = json.load(f)
        return float(pk["bf16_tflops"]), "measured"
    except (OSError, KeyError, ValueError):
        return 1590.0, "fallback"


def traffic_table():
    """Per-launch DRAM bytes of the kernels captured with ncu (committed
    summary, scaled to cells); {kernel: bytes_per_cell} or {}."""
    here = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    path = os.path.join(here, "profiles", "dram_bytes_per_cell.json")
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def roofline(ktimes, ncells, prec):
    """Roofline record of the kernel with the largest total device time."""
    peak, src = peaks()
    best = None
    for name, kt in ktimes.items():
        b = bytes_per_cell(name)
        if b is None or kt["launches"] == 0:
            continue
        if best is None or kt["ms"] > best[1]["ms"]:
            best = (name, kt, b)
    if best is None:
        return None
    name, kt, b = best
    per_launch_ms = kt["ms"] / kt["launches"]
    achieved = b * ncells / (per_launch_ms * 1e-3) / 1e9
    tr = traffic_table().get(name)
    total = sum(k["ms"] for k in ktimes.values())
    return {"kernel": name, "bound": "hbm", "achieved": achieved,
            "peak": peak, "peak_source": src, "unit": "GB/s",
            "frac": achieved / peak,
            "traffic": None if tr is None else tr * ncells,
            "algorithmic_bytes_per_launch": b * ncells,
            "launch_ms": per_launch_ms, "share_of_device_time": kt["ms"] / total}


def step_roofline(ktimes, ncells, steps, step_ms):
    """Whole-step figure: the algorithmic bytes of every full-grid launch in
    ``steps`` steps (coarse multigrid levels, about a seventh more, are not
    counted) over the measured step time."""
    peak, src = peaks()
    total = 0.0
    for name, kt in ktimes.items():
        b = bytes_per_cell(name)
        if b is not None:
            total += b * ncells * kt["launches"]
    per_step = total / max(1, steps)
    achieved = per_step / (step_ms * 1e-3) / 1e9
    return {"bytes_per_step": per_step, "bytes_per_cell": per_step / ncells,
            "achieved": achieved, "peak": peak, "peak_source": src, "unit": "GB/s",
            "frac": achieved / peak}


def closure_case(kind, n, reps=2, device="cuda"):
    """A small seeded case of one closure kernel for profilers (ncu -k ...):
    ``kind`` 'mlp' (the tensor-core MLP closure, pf_mlp_closure) or 'source'
    (the reference's 'source' closure, pf_mlsrc_closure) on an n^3 grid of
    the k0 = 4 spectral field, run ``reps`` times.  Returns the device error
    flag.  Usage:
        python -c "import pyflow_b200.profiling as p; p.closure_case('mlp', 128)"
    """
    import numpy as np
    import torch
    from . import initial as ic
    u, v, w = (t.contiguous() for t in
               ic.spectral_velocity_device((n, n, n), k0=4.0, seed=3, device=device))
    sp = (2 * np.pi / n,) * 3
    if kind == "mlp":
        from . import sfsmodel_mlp as M
        wp = torch.as_tensor(M.pack(M.xavier_init(1))).to(device)
        res = None
        for _ in range(reps):
            res = M.closure(u, v, w, sp, wp, delta=sp[0], out=res[0] if res else None)
        err = res[3]
    elif kind == "source":
        from . import sfsmodel_ML as ML

        class _Geo:
            type = "uniform"
            dx = sp[0]

        class _Dec:
            pass

        class _IC:
            simDt = 0.01

        _Dec.device = torch.device(device)
        torch.manual_seed(0)
        ml = ML.residual_stress(_IC(), _Dec(), _Geo(), model=ML.GatedClosureNet())
        for _ in range(reps):
            ml.update(u, v, w)
        err = ml._err
    else:
        raise ValueError("kind must be 'mlp' or 'source'")
    torch.cuda.synchronize(device)
    return int(err.item())


def slab_case(n, slabs=2, steps=1, device="cuda"):
    """A small seeded case of the x-slab decomposition for profilers (ncu -k
    regex:slab_): ``steps`` FP64 decomposed steps of the k0 = 4 spectral field
    on an n^3 grid split into ``slabs`` slabs on one device (slab.LocalSlabs).
    Returns the last solve's status.  Usage:
        python -c "import pyflow_b200.profiling as p; p.slab_case(192)"
    """
    import numpy as np
    import torch
    from . import initial as ic
    from .slab import LocalSlabs, SlabDomain
    f = [torch.tensor(a, device=device) for a in
         ic.spectral_velocity((n, n, n), k0=4.0, seed=1)]
    D = SlabDomain((n, n, n), (2 * np.pi / n,) * 3, 0.005, 1.0, 0.0025, LocalSlabs(slabs),
                   min_res=1e-10, max_it=20000, poll=8)
    D.set_state(*f)
    info = None
    for _ in range(steps):
        info = D.forward_step()
    torch.cuda.synchronize()
    return info.status


def graph_steps_case(n=512, steps=2, prec="mixed_mg", device="cuda"):
    """Graph-replayed steps of the n^3 decaying-turbulence workload (k0 = 8,
    nu = 0.0012, dt = 0.001, seed 0) for a launch list of the captured path:
    one warm-up step, then ``steps`` steps inside an NVTX range "timed"
    (ncu --nvtx --nvtx-include "timed/" ...).  Returns the plan's statistics.
        python -c "import pyflow_b200.profiling as p; p.graph_steps_case()"
    """
    import numpy as np
    import torch
    from . import initial as ic
    from .plan import StepPlan
    u, v, w = (t.contiguous() for t in
               ic.spectral_velocity_device((n, n, n), k0=8.0, seed=0, device=device))
    p, DP = torch.zeros_like(u), torch.zeros_like(u)
    plan = StepPlan(u, v, w, p, DP, (2 * np.pi / n,) * 3, 0.0012, 1.0, 0.001, min_res=1e-10,
                    max_it=20000, prec=prec)
    plan.launch(1)
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_push("timed")
    plan.launch(steps)
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    st = plan.stats()
    plan.close()
    return st
