"""Generates tests/golden/ref_*.npz: outputs of the REFERENCE ITSELF
(vaishna77/RCS, its unmodified src/*.cpp and tree header compiled against the
project-written Eigen subset by oracle/ref.mk, driven by oracle/ref_driver.cpp
as test/sphere.cpp drives it).  Run in the build container, where the
reference tree is mounted; the fixtures travel, the reference does not.

Cases (the reference's compiled-in frequency, 10 MHz; x-polarised plane wave
of sphere.cpp:172-177):
  s78_l8_t8_f10:   the reference's shipped 78-triangle sphere (117 unknowns),
                   leaf 8, ACA 1e-8, RRQR 1e-10, dense LU solution included;
  s1280_l64_t8_f10: icosphere 3 (1,920 unknowns), the first benchmark
                   configuration's tree (leaf 64, ACA 1e-8, RRQR 1e-10), dense LU
                   solution included;
  s1280_l8_t5_f7:  the same mesh at the large benchmark's tolerances (ACA 1e-5,
                   RRQR 1e-7) with leaf 8: about 1,250 fill-in recompressions;
  s1280_l3_t5_f7:  the same with leaf 3: three levels, so the non-leaf
                   elimination and the level-to-level basis updates run.

Each file holds the right-hand side, the dense LU and AIFMM solutions, 4,096
seeded matrix entries, every box's rank after assembly and after
factorization, the reference's timings, and the shape and Frobenius norm of
every box's L2P, P2M and L2M_f blocks after assembly and after
factorization.

Usage: python tests/golden/make_ref_golden.py [reference_root] [threads]
"""
from __future__ import annotations

import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from rcs_b200 import mesh as M  # noqa: E402

CASES = {
    "s78_l8_t8_f10": dict(mesh="shipped78", leaf=8, tol=8, ftol=10, dense=1),
    "s1280_l64_t8_f10": dict(mesh=3, leaf=64, tol=8, ftol=10, dense=1),
    "s1280_l8_t5_f7": dict(mesh=3, leaf=8, tol=5, ftol=7, dense=0),
    "s1280_l3_t5_f7": dict(mesh=3, leaf=3, tol=5, ftol=7, dense=0),
}


def read_output(path: str) -> dict:
    """The binary layout written by oracle/ref_driver.cpp."""
    b = open(path, "rb").read()
    o = 0

    def take(dt, n):
        nonlocal o
        v = np.frombuffer(b, dt, n, o).copy()
        o += np.dtype(dt).itemsize * n
        return v

    magic, n, n_levels, n_pairs = take(np.int32, 4)
    assert magic == 0x52454631, "not an aifmm_ref output"
    out = dict(N=int(n), nLevels=int(n_levels), rhs=take(np.complex128, n), x_lu=take(np.complex128, n),
               x=take(np.complex128, n))
    ij = np.zeros((n_pairs, 2), np.int32)
    ent = np.zeros(n_pairs, np.complex128)
    for q in range(n_pairs):
        ij[q] = take(np.int32, 2)
        ent[q] = take(np.complex128, 1)[0]
    out["pairs"], out["entries"] = ij, ent
    n_boxes = sum(8 ** j for j in range(int(n_levels) + 1))
    rk = take(np.int32, 2 * n_boxes).reshape(-1, 2)
    out["rank_assembled"], out["rank_factored"] = rk[:, 0], rk[:, 1]
    out["t_assemble"], out["t_factor"], out["t_solve"] = take(np.float64, 3)
    for key in ("blocks_assembled", "blocks_factored"):
        cnt = int(take(np.int64, 1)[0])
        out[key] = take(np.float64, 7 * cnt).reshape(cnt, 7)
    assert o == len(b), "trailing bytes in an aifmm_ref output"
    return out


def main(ref_root: str, threads: int) -> None:
    subprocess.run(["make", "-s", "-f", os.path.join(ROOT, "oracle", "ref.mk"), f"REF={ref_root}", "-j8"], check=True,
                   cwd=ROOT)
    exe = os.path.join(ROOT, "oracle", "_ref", "aifmm_ref")
    with tempfile.TemporaryDirectory() as tmp:
        for name, c in CASES.items():
            if c["mesh"] == "shipped78":
                d = os.path.join(ref_root, "inputFiles", "radius015")
                nf, pf = os.path.join(d, "nodeList78.txt"), os.path.join(d, "patchList78.txt")
                m = M.read_mesh(nf, pf)
            else:
                m = M.icosphere(c["mesh"], 0.15)
                nf, pf = os.path.join(tmp, "nodes.txt"), os.path.join(tmp, "patches.txt")
                M.write_mesh(m, nf, pf)
            binp = os.path.join(tmp, name + ".bin")
            subprocess.run([exe, "EFIE", nf, pf, str(c["leaf"]), str(c["tol"]), str(c["ftol"]), binp, str(c["dense"]),
                            str(threads)], check=True, cwd=tmp, stdout=subprocess.DEVNULL)
            r = read_output(binp)
            for key in ("blocks_assembled", "blocks_factored"):  # the bases and L2M_f of every box
                t = r[key]
                r[key] = t[np.isin(t[:, 2], (0, 1, 9))]
            path = os.path.join(HERE, f"ref_{name}.npz")
            np.savez_compressed(path, nodes=m.nodes, tris=m.tris, freq=1.0e7, leaf=c["leaf"], tol_pow=c["tol"],
                                fillin_tol=c["ftol"], dense=c["dense"], **r)
            print("wrote", path, "N", r["N"], "levels", r["nLevels"], "factor s", round(float(r["t_factor"]), 2),
                  flush=True)


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("AIFMM_REFERENCE_ROOT", "")
    if not root:
        sys.exit("usage: make_ref_golden.py <reference tree> [threads] (or set AIFMM_REFERENCE_ROOT)")
    main(root, int(sys.argv[2]) if len(sys.argv) > 2 else 4)
