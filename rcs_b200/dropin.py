"""Compiler flags for C++ drivers written against the reference's class API.

The headers under include/aifmm/ (AIFMM.hpp, EFIEMatrix.hpp, ACA.hpp, rrqr.hpp,
... and a project-written Eigen subset) sit over libaifmm_b200.so.  A driver
such as the reference's test/sphere.cpp builds unchanged with

    g++ -std=c++17 -fopenmp $(python -m rcs_b200.dropin --cflags) sphere.cpp \\
        $(python -m rcs_b200.dropin --libs) -o sphere

Usage: python -m rcs_b200.dropin [--cflags] [--libs]
"""
from __future__ import annotations

import argparse
import os
import subprocess
from typing import Sequence

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
INCLUDE = os.path.join(ROOT, "include", "aifmm")
LIB_DIR = os.path.join(HERE, "lib")


def cflags(defines: Sequence[str] = ("USE_COMPLEX64", "USE_THREE")) -> list[str]:
    return ["-std=c++17", *[f"-D{d}" for d in defines], "-I", INCLUDE]


def libs() -> list[str]:
    return ["-L", LIB_DIR, "-laifmm_b200", f"-Wl,-rpath,{LIB_DIR}"]


def compile_driver(sources: Sequence[str], out: str, defines: Sequence[str] = ("USE_COMPLEX64", "USE_THREE"),
                   extra: Sequence[str] = (), link: bool = True) -> subprocess.CompletedProcess:
    """g++ a driver against the drop-in headers (and the library when link)."""
    cmd = ["g++", "-O1", "-Wall", *cflags(defines), *extra, *sources, "-o", out]
    if link:
        cmd += libs()
    else:
        cmd = ["g++", "-fsyntax-only", "-Wall", *cflags(defines), *extra, *sources]
    return subprocess.run(cmd, capture_output=True, text=True)


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--cflags", action="store_true")
    ap.add_argument("--libs", action="store_true")
    a = ap.parse_args()
    parts = []
    if a.cflags or not a.libs:
        parts += cflags()
    if a.libs:
        parts += libs()
    print(" ".join(parts))


if __name__ == "__main__":
    main()
