"""ctypes binding of libpyflow_b200.so (C ABI: include/pyflow_b200.h).

The shared library is the only compute path: importing this module without the
library raises, and there is no CPU fallback.  Build it with
``python pyflow-public_b200/csrc/build.py`` (or ``__graft_entry__.build()``).
"""
import ctypes
import os

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libpyflow_b200.so")

PF_OK, PF_ERR_BAD_ARG, PF_ERR_CUDA, PF_BREAKDOWN, PF_MAXIT, PF_NONFINITE, \
    PF_STAGNATION, PF_ERR_TOO_LARGE = range(8)
PF_FP64, PF_MIXED, PF_MIXED_MG = 0, 1, 2
PF_WARM_START = 0x100   # flag in prec: mixed solves start from the DP given


class Grid(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
                ("dx", ctypes.c_double), ("dy", ctypes.c_double),
                ("dz", ctypes.c_double)]


class SolveInfo(ctypes.Structure):
    _fields_ = [("max_res", ctypes.c_double), ("iterations", ctypes.c_int),
                ("outer", ctypes.c_int), ("status", ctypes.c_int)]


class PyFlowError(RuntimeError):
    """A pf_* entry point returned an error status."""

    def __init__(self, fn, status):
        self.status = status
        super().__init__("%s failed: %s (status %d)" % (
            fn, _lib.pf_status_string(status).decode(), status))


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            "libpyflow_b200.so not found at %s; build it with "
            "`python pyflow-public_b200/csrc/build.py`" % LIB_PATH)
    L = ctypes.CDLL(LIB_PATH)
    P, D, I, S = ctypes.c_void_p, ctypes.c_double, ctypes.c_int, ctypes.c_size_t
    G = ctypes.POINTER(Grid)
    sigs = {
        "pf_version": ([], I),
        "pf_status_string": ([I], ctypes.c_char_p),
        "pf_workspace_bytes": ([G, I], S),
        "pf_rhs_ns": ([G, I, P, P, P, P, D, D, P, P, P, P, P], I),
        "pf_div_vel": ([G, P, P, P, P, P], I),
        "pf_laplace_apply": ([G, P, P, P], I),
        "pf_predictor_step": ([G, I, I, P, P, P, P, D, D, P, D, P, S, P], I),
        "pf_bicgstab_solve": ([G, I, D, D, D, I, P, P, P, P, S, P,
                               ctypes.POINTER(SolveInfo)], I),
        "pf_jacobi_solve": ([G, D, D, I, P, P, P, P, S, P,
                             ctypes.POINTER(ctypes.c_double)], I),
        "pf_vel_corr": ([G, P, D, P, P, P, P], I),
        "pf_forward_step": ([G, I, I, I, P, P, P, P, P, P, D, D, P, D, D, I, P,
                             S, P, ctypes.POINTER(SolveInfo)], I),
        "pf_stats": ([G, P, P, P, P, P, S, P], I),
        "pf_flow_stats": ([G, P, P, P, D, P, P, S, P], I),
        "pf_sgs_closure": ([G, I, P, P, P, D, P, P], I),
        "pf_mlp_pack_bytes": ([], S),
        "pf_restart_pack": ([G, P, P, P], I),
        "pf_restart_unpack": ([G, P, P, P], I),
        "pf_mlp_closure": ([G, P, P, P, P, P, P, P, P], I),
        "pf_mlp_scales_workspace_bytes": ([], S),
        "pf_mlp_scales": ([G, P, P, P, D, P, P, S, P], I),
        "pf_mlsrc_pack_bytes": ([], S),
        "pf_mlsrc_workspace_bytes": ([G], S),
        "pf_mlsrc_pack": ([ctypes.POINTER(ctypes.c_void_p), P, P], I),
        "pf_mlsrc_closure": ([G, P, P, P, P, P, P, P, S, P, P], I),
    }
    for name, (args, res) in sigs.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = res
    return L


_lib = _load()


def lib():
    return _lib


def check(fn_name, status):
    if status != PF_OK:
        raise PyFlowError(fn_name, status)
