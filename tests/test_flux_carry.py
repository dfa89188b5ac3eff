"""The RK4 stage kernels compute each face's flux terms once: a cell's x-minus
terms are carried from the cell before it along the x march (XFace), its y- and
z-minus terms are the plus-face terms of its neighbours (YFace, ZFace; the face
form of pf_flux.cuh).  This CPU test compiles the same per-cell routines for the
host (tests/flux_carry_check.cpp) and checks that both forms agree bit for bit
with the full evaluation (rhs_core) in FP64 and FP32 on small random periodic
grids."""
import os
import shutil
import subprocess

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_x_face_carry_is_bit_identical(tmp_path):
    cxx = shutil.which("g++") or shutil.which("c++")
    if cxx is None:
        pytest.skip("no host C++ compiler")
    exe = tmp_path / "flux_carry_check"
    subprocess.run([cxx, "-std=c++17", "-O2", "-ffp-contract=off",
                    "-I", os.path.join(REPO, "pyflow-public_b200", "csrc"),
                    os.path.join(REPO, "tests", "flux_carry_check.cpp"), "-o", str(exe)],
                   check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "mismatches fp64 0 fp32 0" in r.stdout
    assert "face mismatches fp64 0 fp32 0" in r.stdout
