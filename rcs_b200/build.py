"""Builds libaifmm_b200.so in-tree (rcs_b200/lib/) with nvcc for sm_100a.

Usage: python -m rcs_b200.build [--force] [--verbose]
The build cross-compiles without a GPU.  Objects go to rcs_b200/lib/_build/
and are rebuilt when a source or header is newer than the object.
"""
from __future__ import annotations

import argparse
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "csrc")
LIB_DIR = os.path.join(HERE, "lib")
OBJ_DIR = os.path.join(LIB_DIR, "_build")
LIB = os.path.join(LIB_DIR, "libaifmm_b200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr", "-I", INCLUDE,
          "-Xptxas", "-warn-spills"]
# Files whose FP64 arithmetic must round like the reference: no a*b+c fusion.
NO_FMA = {"assemble.cu", "lowrank.cu", "farfield.cu", "mesh_build.cu"}


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _newest_header() -> float:
    hs = glob.glob(os.path.join(SRC, "*.cuh")) + glob.glob(os.path.join(SRC, "*.h")) + \
        glob.glob(os.path.join(INCLUDE, "*.h"))
    return max((os.path.getmtime(h) for h in hs), default=0.0)


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(OBJ_DIR, exist_ok=True)
    sources = sorted(glob.glob(os.path.join(SRC, "*.cu")) + glob.glob(os.path.join(SRC, "*.cpp")))
    hdr = _newest_header()
    objs = []
    rebuilt = False
    nv = nvcc()
    for s in sources:
        name = os.path.basename(s)
        o = os.path.join(OBJ_DIR, name + ".o")
        objs.append(o)
        if not force and os.path.exists(o) and os.path.getmtime(o) >= max(os.path.getmtime(s), hdr):
            continue
        flags = list(COMMON)
        if name in NO_FMA:
            flags += ["-fmad=false"]
        cmd = [nv, *ARCH, *flags, "-c", s, "-o", o]
        if name.endswith(".cpp"):
            cmd = [nv, *flags, "-x", "cu", *ARCH, "-c", s, "-o", o]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError(f"nvcc failed on {name}")
        if verbose and r.stderr.strip():
            sys.stderr.write(r.stderr)
        rebuilt = True
    if rebuilt or force or not os.path.exists(LIB):
        cmd = [nv, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart", "-lcuda"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("link failed")
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args()
    print(build(a.force, a.verbose))
