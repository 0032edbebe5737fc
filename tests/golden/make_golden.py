"""Generates the committed golden fixtures of tests/golden/ (run in the build
container, where the reference tree is mounted; the GPU box never runs this).

sphere78.npz: the reference's only shipped geometry (inputFiles/radius015,
78 triangles, 117 RWG unknowns) with the CPU oracle's outputs on it at the
reference's hard-coded 10 MHz: a sample of matrix entries, the reference RHS
(EFIEMatrix::getRhs with Einc = x), the dense-LU solution and the AIFMM
solution with the driver's tolerances.

Usage: python tests/golden/make_golden.py [reference_root]
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from rcs_b200 import mesh as M  # noqa: E402


def main(ref_root: str) -> None:
    d = os.path.join(ref_root, "inputFiles", "radius015")
    m = M.read_mesh(os.path.join(d, "nodeList78.txt"), os.path.join(d, "patchList78.txt"))
    K = oracle.EFIE(m, 1.0e7)
    A = K.dense()
    b = K.rhs_reference((1.0, 0.0, 0.0))
    x_lu = K.dense_solve(b)
    S = oracle.AIFMM(K, leaf_size=8, tol_pow=8, fillin_tol=10)
    S.factorize()
    x_h = S.solve(b)
    rwg, ln = K.rwg()
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "sphere78.npz")
    np.savez_compressed(out, nodes=m.nodes, tris=m.tris, freq=1.0e7, A=A, rhs=b, x_lu=x_lu, x_aifmm=x_h,
                        rwg=rwg, length=ln, locations=K.locations())
    print("wrote", out, A.shape)


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("AIFMM_REFERENCE_ROOT", "")
    if not root:
        sys.exit("usage: make_golden.py <reference tree> (or set AIFMM_REFERENCE_ROOT)")
    main(root)
