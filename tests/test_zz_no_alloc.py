"""pf_bicgstab_solve_noalloc: the BiCGStab solve for callers that cannot
allocate device memory (its scratch is a fixed array inside the library).

Called through the C ABI with ctypes; its results must match the workspace
entry point pf_bicgstab_solve within the BiCGStab tolerance the other parity
tests use, on two calls in a row (the shared scratch keeps the previous call's
contents, so the second call checks that nothing stale leaks in).  This file
is named to be collected last.
"""
import ctypes
import os

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(REPO, "pyflow-public_b200", "libpyflow_b200.so")


class Grid(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
                ("dx", ctypes.c_double), ("dy", ctypes.c_double),
                ("dz", ctypes.c_double)]


class Info(ctypes.Structure):
    _fields_ = [("max_res", ctypes.c_double), ("iterations", ctypes.c_int),
                ("outer", ctypes.c_int), ("status", ctypes.c_int)]


@pytest.fixture(scope="module")
def lib():
    L = ctypes.CDLL(LIB)
    P, D, I, S = ctypes.c_void_p, ctypes.c_double, ctypes.c_int, ctypes.c_size_t
    L.pf_workspace_bytes.argtypes = [ctypes.POINTER(Grid), I]
    L.pf_workspace_bytes.restype = S
    L.pf_bicgstab_solve.argtypes = [ctypes.POINTER(Grid), I, D, D, D, I, P, P, P,
                                    P, S, P, ctypes.POINTER(Info)]
    L.pf_bicgstab_solve.restype = I
    L.pf_bicgstab_solve_noalloc.argtypes = [ctypes.POINTER(Grid), D, D, D, I, P,
                                            P, P, P, ctypes.POINTER(Info)]
    L.pf_bicgstab_solve_noalloc.restype = I
    return L


def _source(shape, seed):
    """Divergence of a random staggered field: a consistent Poisson RHS."""
    rng = np.random.default_rng(seed)
    u, v, w = (rng.standard_normal(shape) for _ in range(3))
    h = (0.2, 0.2, 0.2)
    d = ((np.roll(u, -1, 0) - u) / h[0] + (np.roll(v, -1, 1) - v) / h[1]
         + (np.roll(w, -1, 2) - w) / h[2])
    return d, h


def _solve(lib, noalloc, src, grid, stream, check_no_alloc=False):
    DP = torch.zeros_like(src)
    p = torch.zeros_like(src)
    info = Info()
    torch.cuda.synchronize()
    before = (torch.cuda.mem_get_info()[0], torch.cuda.memory_reserved())
    args = (ctypes.byref(grid),)
    if noalloc:
        rc = lib.pf_bicgstab_solve_noalloc(
            ctypes.byref(grid), 1.0, 0.01, 1e-10, 2000, src.data_ptr(),
            DP.data_ptr(), p.data_ptr(), stream, ctypes.byref(info))
    else:
        need = lib.pf_workspace_bytes(*args, 0)
        ws = torch.empty(need, dtype=torch.uint8, device=src.device)
        rc = lib.pf_bicgstab_solve(
            ctypes.byref(grid), 0, 1.0, 0.01, 1e-10, 2000, src.data_ptr(),
            DP.data_ptr(), p.data_ptr(), ws.data_ptr(), ws.numel(), stream,
            ctypes.byref(info))
    torch.cuda.synchronize()
    assert rc == 0, rc
    if check_no_alloc:
        # neither the device's free memory nor torch's pool moved: the call
        # allocated nothing
        assert (torch.cuda.mem_get_info()[0], torch.cuda.memory_reserved()) == before
    return DP.cpu().numpy(), p.cpu().numpy(), info


def test_noalloc_matches_workspace_entry_point_twice(lib):
    stream = torch.cuda.current_stream().cuda_stream
    for call, (shape, seed) in enumerate((((40, 32, 48), 3), ((64, 64, 64), 4))):
        d, h = _source(shape, seed)
        src = torch.tensor(d, device="cuda")
        grid = Grid(*shape, *h)
        ref_DP, ref_p, ref_info = _solve(lib, False, src, grid, stream)
        # the first call in the process may load device code; from the second
        # call on, the free device memory must not change across a call
        DP, p, info = _solve(lib, True, src, grid, stream, check_no_alloc=call > 0)
        assert info.status == 0 and ref_info.status == 0, call
        assert info.max_res <= 1e-10
        assert abs(info.iterations - ref_info.iterations) <= max(2, ref_info.iterations // 10)
        scale = np.abs(ref_DP).max()
        assert np.abs(DP - ref_DP).max() <= 2e-8 * scale, call
        assert np.abs(p - ref_p).max() <= 2e-8 * scale, call


def test_noalloc_rejects_grids_above_limit(lib):
    grid = Grid(65, 64, 64, 0.1, 0.1, 0.1)
    t = torch.zeros(8, dtype=torch.float64, device="cuda")
    info = Info()
    rc = lib.pf_bicgstab_solve_noalloc(
        ctypes.byref(grid), 1.0, 0.01, 1e-10, 10, t.data_ptr(), t.data_ptr(),
        t.data_ptr(), None, ctypes.byref(info))
    assert rc == 7  # PF_ERR_TOO_LARGE
