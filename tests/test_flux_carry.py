"""The RK4 stage kernels march along x and take each cell's x-minus flux terms
from the x-plus terms of the cell before it (pf_flux.cuh, XFace).  This CPU
test compiles the same per-cell routine for the host (tests/flux_carry_check.cpp)
and checks that the carried march and the full evaluation agree bit for bit in
FP64 and FP32 on small random periodic grids."""
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
    assert "fp64 0 fp32 0" in r.stdout
