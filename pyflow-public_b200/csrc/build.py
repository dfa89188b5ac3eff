"""Build libpyflow_b200.so (sm_100a) in-tree with nvcc.

    python pyflow-public_b200/csrc/build.py [--force] [--verbose]

Every .cu file in this directory is compiled with
``-gencode arch=compute_100a,code=sm_100a -lineinfo --fmad=false`` (no FMA
contraction: FP64 operators then round exactly like the reference's torch
ops; fused multiply-adds are explicit fma() calls) and linked into
``pyflow-public_b200/libpyflow_b200.so``.  The library links only the CUDA
runtime (no torch), so any host language can load it.
"""
import argparse
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
OUT = os.path.join(PKG, "libpyflow_b200.so")
OBJ = os.path.join(PKG, "_build")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--fmad=false", "-Xcompiler", "-fPIC",
         "-Xcompiler", "-Wall", "--expt-relaxed-constexpr"]


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc",
                 shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(glob.glob(os.path.join(HERE, "*.cu")))


def deps():
    return sources() + sorted(glob.glob(os.path.join(HERE, "*.cuh"))) + [
        os.path.join(os.path.dirname(PKG), "include", "pyflow_b200.h")]


def up_to_date():
    if not os.path.exists(OUT):
        return False
    t = os.path.getmtime(OUT)
    return all(os.path.getmtime(f) <= t for f in deps())


def build(force=False, verbose=False, ptxas_info=False):
    if not force and up_to_date():
        return OUT
    os.makedirs(OBJ, exist_ok=True)
    nv = nvcc()
    extra = ["-Xptxas", "-v"] if ptxas_info else []
    jobs = []
    for src in sources():
        obj = os.path.join(OBJ, os.path.basename(src)[:-3] + ".o")
        cmd = [nv, *ARCH, *FLAGS, *extra, "-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd))
        # the translation units are independent: compile them concurrently
        jobs.append((src, obj, subprocess.Popen(cmd, stdout=subprocess.PIPE,
                                                stderr=subprocess.PIPE, text=True)))
    objs, failed = [], None
    for src, obj, proc in jobs:
        out, err = proc.communicate()
        if proc.returncode != 0:
            sys.stderr.write(out + err)
            failed = failed or src
        elif ptxas_info or verbose:
            sys.stderr.write(err)
        objs.append(obj)
    if failed:
        raise RuntimeError("nvcc failed on " + failed)
    cmd = [nv, *ARCH, "-shared", "-o", OUT + ".tmp", *objs, "-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("link failed")
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-info", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose, ptxas_info=a.ptxas_info))
