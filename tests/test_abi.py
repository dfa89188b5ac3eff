"""The C-ABI library loads without a GPU and exports every entry point that
include/pyflow_b200.h declares (no compute calls here)."""
import ctypes
import os
import re

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(REPO, "include", "pyflow_b200.h")
LIB = os.path.join(REPO, "pyflow-public_b200", "libpyflow_b200.so")


def declared():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(pf_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_entry_points():
    names = declared()
    assert "pf_bicgstab_solve" in names and "pf_forward_step" in names


def test_library_exports_all_declared_symbols():
    if not os.path.exists(LIB):
        pytest.skip("library not built (run __graft_entry__.build())")
    lib = ctypes.CDLL(LIB)
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_host_only_calls():
    if not os.path.exists(LIB):
        pytest.skip("library not built")
    lib = ctypes.CDLL(LIB)
    assert lib.pf_version() >= 100
    lib.pf_status_string.restype = ctypes.c_char_p
    assert lib.pf_status_string(0) == b"ok"

    class Grid(ctypes.Structure):
        _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int),
                    ("nz", ctypes.c_int), ("dx", ctypes.c_double),
                    ("dy", ctypes.c_double), ("dz", ctypes.c_double)]

    lib.pf_workspace_bytes.restype = ctypes.c_size_t
    lib.pf_workspace_bytes.argtypes = [ctypes.POINTER(Grid), ctypes.c_int]
    g = Grid(64, 64, 64, 0.1, 0.1, 0.1)
    n64 = lib.pf_workspace_bytes(ctypes.byref(g), 0)
    assert n64 >= 8 * 64 ** 3 * 8
    bad = Grid(0, 64, 64, 0.1, 0.1, 0.1)
    assert lib.pf_workspace_bytes(ctypes.byref(bad), 0) == 0
    # argument validation happens before any CUDA call
    lib.pf_div_vel.restype = ctypes.c_int
    assert lib.pf_div_vel(ctypes.byref(g), None, None, None, None, None) == 1


def test_step_plan_workspace_sizes():
    """The step plan's workspace (host arithmetic only): the multigrid form
    holds the mixed form's vectors plus a 256-byte aligned slot for the
    coarsest level's pseudo-inverse (64 x 64 FP32), which the plan computes
    once instead of in every step."""
    if not os.path.exists(LIB):
        pytest.skip("library not built")
    lib = ctypes.CDLL(LIB)

    class Grid(ctypes.Structure):
        _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int),
                    ("nz", ctypes.c_int), ("dx", ctypes.c_double),
                    ("dy", ctypes.c_double), ("dz", ctypes.c_double)]

    lib.pf_step_plan_workspace_bytes.restype = ctypes.c_size_t
    lib.pf_step_plan_workspace_bytes.argtypes = [ctypes.POINTER(Grid), ctypes.c_int]
    for shape in ((64, 64, 64), (24, 20, 36), (33, 17, 70)):
        g = Grid(*shape, 0.1, 0.1, 0.1)
        fp64, mixed, mg = (lib.pf_step_plan_workspace_bytes(ctypes.byref(g), pr)
                           for pr in (0, 1, 2))
        n = shape[0] * shape[1] * shape[2]
        assert fp64 >= 9 * 8 * n and mixed >= 12 * 8 * n
        # the coarsest level's pseudo-inverse and the grid-barrier words
        assert mg == mixed + 64 * 64 * 4 + 256
        assert mg % 256 == 0 and mixed % 256 == 0


def test_step_closure_sizes_and_argument_checks():
    """pf_step_closure_bytes: one field (Smagorinsky viscosity) or six
    (gradient-model stresses) in the stages' type; for the MLP a scratch of
    scales and reduction partials, the six FP64 stresses and, for the mixed
    forms, their float copy, each 256-byte aligned.  pf_step_plan_create_sfs
    rejects an unknown closure, a short or misaligned closure buffer and an
    MLP closure without its network before any CUDA call."""
    if not os.path.exists(LIB):
        pytest.skip("library not built")
    lib = ctypes.CDLL(LIB)

    class Grid(ctypes.Structure):
        _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int),
                    ("nz", ctypes.c_int), ("dx", ctypes.c_double),
                    ("dy", ctypes.c_double), ("dz", ctypes.c_double)]

    class Closure(ctypes.Structure):
        _fields_ = [("kind", ctypes.c_int), ("coef", ctypes.c_double),
                    ("wpack", ctypes.c_void_p), ("err", ctypes.c_void_p),
                    ("field", ctypes.c_void_p), ("field_bytes", ctypes.c_size_t)]

    for fn in (lib.pf_step_closure_bytes, lib.pf_step_closure_stage_offset):
        fn.restype = ctypes.c_size_t
        fn.argtypes = [ctypes.POINTER(Grid), ctypes.c_int, ctypes.c_int]
    g = Grid(24, 20, 36, 0.1, 0.1, 0.1)
    n = 24 * 20 * 36
    a256 = lambda b: (b + 255) // 256 * 256  # noqa: E731
    by = lambda pr, k: lib.pf_step_closure_bytes(ctypes.byref(g), pr, k)  # noqa: E731
    off = lambda pr, k: lib.pf_step_closure_stage_offset(ctypes.byref(g), pr, k)  # noqa: E731
    assert by(0, 1) == 8 * n and by(0, 2) == 6 * 8 * n
    assert by(2, 1) == 4 * n and by(1, 2) == 6 * 4 * n
    assert off(0, 1) == off(2, 2) == 0
    scratch = a256(256 + 256 + 1024 * 8)
    assert off(0, 3) == scratch and by(0, 3) == scratch + a256(48 * n)
    assert off(2, 3) == scratch + a256(48 * n) and by(2, 3) == off(2, 3) + a256(24 * n)
    assert by(0, 4) == 0 and by(0, 0) == 0
    P, D, I, S = ctypes.c_void_p, ctypes.c_double, ctypes.c_int, ctypes.c_size_t
    lib.pf_step_plan_create_sfs.restype = I
    lib.pf_step_plan_create_sfs.argtypes = [ctypes.POINTER(Grid), I, I] + [P] * 5 + [D] * 4 + [
        I, ctypes.POINTER(Closure), P, S, P, ctypes.POINTER(P)]
    fake = 1 << 20  # never dereferenced: every call below fails its checks first
    h = P(0)

    def create(kind, field, nbytes, wpack=fake, err=fake):
        c = Closure(kind, 0.001, wpack, err, field, nbytes)
        return lib.pf_step_plan_create_sfs(
            ctypes.byref(g), 0, 1, fake, fake, fake, fake, fake, 0.01, 1.0, 0.001, 1e-10, 100,
            ctypes.byref(c), fake, 1 << 30, fake, ctypes.byref(h))

    assert create(4, fake, 6 * 8 * n) == 1
    assert create(1, fake, 8 * n - 8) == 1
    assert create(1, fake + 16, 8 * n) == 1
    assert create(2, None, 6 * 8 * n) == 1
    assert create(3, fake, by(0, 3), wpack=None) == 1
    assert create(3, fake, by(0, 3), err=None) == 1
    assert create(3, fake, by(0, 3) - 256) == 1
    assert h.value is None
    lib.pf_mlp_scales_workspace_bytes.restype = S
    assert lib.pf_mlp_scales_workspace_bytes() == 256 + 1024 * 8


def test_struct_layouts_match_the_header(tmp_path):
    """The ctypes structures the Python side passes across the ABI have the
    C compiler's layout of the header's structs (size and every field
    offset): pf_grid, pf_solve_info, pf_step_closure, pf_batch_member."""
    import shutil
    import subprocess
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    src = tmp_path / "layout.c"
    fields = {
        "pf_grid": ["nx", "ny", "nz", "dx", "dy", "dz"],
        "pf_solve_info": ["max_res", "iterations", "outer", "status"],
        "pf_step_closure": ["kind", "coef", "wpack", "err", "field", "field_bytes"],
        "pf_batch_member": ["grid", "u", "v", "w", "p", "DP", "mu", "rho", "dt", "min_res",
                            "max_it", "fresh", "ws", "ws_bytes", "stats"],
    }
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "pyflow_b200.h"',
             "int main(void) {"]
    for st, fs in fields.items():
        lines.append('printf("%s size %%zu\\n", sizeof(%s));' % (st, st))
        for f in fs:
            lines.append('printf("%s %s %%zu\\n", offsetof(%s, %s));' % (st, f, st, f))
    lines.append("return 0; }")
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run([cc, "-I", os.path.join(REPO, "include"), str(src), "-o", str(exe)],
                   check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout
    got = {tuple(ln.split()[:2]): int(ln.split()[2]) for ln in out.splitlines()}
    if not os.path.exists(LIB):
        pytest.skip("library not built")
    import pyflow_b200._lib as L
    from pyflow_b200.plan import BatchMember, StepClosure
    py = {"pf_grid": L.Grid, "pf_solve_info": L.SolveInfo, "pf_step_closure": StepClosure,
          "pf_batch_member": BatchMember}
    for st, cls in py.items():
        assert ctypes.sizeof(cls) == got[(st, "size")], st
        for f in fields[st]:
            assert getattr(cls, f).offset == got[(st, f)], (st, f)


def _c_args(decl):
    """Argument types of a prototype's parameter list, as (kind, stars,
    base type) with kind 'ptr', 'int', 'double', 'size_t' or 'void'."""
    decl = decl.strip()
    if decl in ("", "void"):
        return []
    out = []
    for a in decl.split(","):
        toks = a.replace("*", " * ").split()
        stars = toks.count("*")
        base = [t for t in toks[:-1] if t not in ("const", "*")]
        base = base[0] if base else ""
        if stars:
            out.append(("ptr", stars, base))
        else:
            out.append(({"int": "int", "double": "double", "size_t": "size_t"}.get(base, base),
                        0, base))
    return out


def test_python_signatures_match_the_header():
    """Every entry point the Python side registers (argtypes / restype) has
    the header's parameter count and scalar types; pointer parameters are
    passed as pointers."""
    if not os.path.exists(LIB):
        pytest.skip("library not built")
    import pyflow_b200._lib as L
    import pyflow_b200.adjoint  # noqa: F401  (registers the adjoint entry points)
    import pyflow_b200.plan  # noqa: F401  (registers the plan entry points)
    import pyflow_b200.profiling  # noqa: F401
    import pyflow_b200.slab  # noqa: F401
    src = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    protos = re.findall(r"([A-Za-z_][\w\s\*]*?)\s*\b(pf_[a-z0-9_]+)\s*\(([^)]*)\)\s*;", src)
    lib = L.lib()
    scalar = {"int": ctypes.c_int, "double": ctypes.c_double, "size_t": ctypes.c_size_t}
    checked = 0
    for ret, name, args in protos:
        fn = getattr(lib, name)
        if fn.argtypes is None:
            continue
        want = _c_args(args)
        assert len(fn.argtypes) == len(want), name
        for i, ((kind, stars, base), got) in enumerate(zip(want, fn.argtypes)):
            if kind == "ptr":
                assert got in (ctypes.c_void_p, ctypes.c_char_p) or hasattr(got, "_type_") \
                    and not isinstance(got._type_, str), (name, i, base)
            else:
                assert got is scalar[kind], (name, i, base, got)
        r = ret.replace("const", "").split()
        if "*" in ret:
            assert fn.restype in (ctypes.c_char_p, ctypes.c_void_p), name
        elif r and r[-1] in scalar:
            assert fn.restype is scalar[r[-1]], (name, fn.restype)
        checked += 1
    assert checked >= 30, checked
