"""Generates tests/golden/sphere7680_c3tol.npz: the CPU oracle's AIFMM
solutions on the 7,680-unknown sphere (icosphere 4, R = 0.15 m, f = 4 GHz)
at the tolerances of the 122,880-unknown benchmark (ACA 1e-5, RRQR 1e-7),
for two tree shapes, plus the oracle's dense-LU solution of the same system.
The oracle takes minutes at this size, so the GPU parity tests read these
outputs instead of running it.  No reference files are read.

Shapes:
  leaf128: leaf size 128, the reference's depth rule (2 levels, about 137
           unknowns per leaf: the largest leaves at this N);
  lvl3:    3 levels, the benchmark's depth (about 28 unknowns per leaf).
Right-hand sides: two seeded plane waves (the benchmark's generator).

Usage: python tests/golden/make_c3tol.py [threads]
"""
from __future__ import annotations

import math
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from rcs_b200 import mesh as M  # noqa: E402

SUB, RADIUS, FREQ, TOL, FTOL = 4, 0.15, 4.0e9, 5, 7
SHAPES = {"leaf128": dict(leaf=128, levels=0), "lvl3": dict(leaf=8, levels=3)}


def plane_waves(n: int, seed: int = 4):
    """Seeded incidence directions uniform on the sphere, alternating
    theta/phi polarisation (the benchmark's generator)."""
    rng = np.random.Generator(np.random.MT19937(seed))
    out = []
    for q in range(n):
        th = math.acos(1 - 2 * rng.random())
        ph = 2 * math.pi * rng.random()
        k = np.array([math.sin(th) * math.cos(ph), math.sin(th) * math.sin(ph), math.cos(th)])
        e_th = np.array([math.cos(th) * math.cos(ph), math.cos(th) * math.sin(ph), -math.sin(th)])
        e_ph = np.array([-math.sin(ph), math.cos(ph), 0.0])
        out.append((k, (e_th if q % 2 == 0 else e_ph).astype(np.complex128)))
    return out


def main(threads: int) -> None:
    oracle.set_threads(threads)
    m = M.icosphere(SUB, RADIUS)
    K = oracle.EFIE(m, FREQ)
    B = np.stack([K.rhs_plane(k, e) for k, e in plane_waves(2)], axis=1)
    out = dict(sub=SUB, radius=RADIUS, freq=FREQ, tol_pow=TOL, fillin_tol=FTOL, rhs=B)
    for name, sh in SHAPES.items():
        t0 = time.perf_counter()
        S = oracle.AIFMM(K, leaf_size=sh["leaf"], tol_pow=TOL, fillin_tol=FTOL, n_levels=sh["levels"])
        t1 = time.perf_counter()
        S.factorize()
        t2 = time.perf_counter()
        X = np.stack([S.solve(B[:, q]) for q in range(B.shape[1])], axis=1)
        info = S.info()
        print(name, "assemble", round(t1 - t0, 1), "factor", round(t2 - t1, 1), "s", info, flush=True)
        out[f"{name}_leaf"] = sh["leaf"]
        out[f"{name}_levels"] = sh["levels"]
        out[f"{name}_x"] = X
        for key in ("nLevels", "startLevel", "avgLeafSize", "avgMultipoles", "maxRank", "nRRQR", "nCompressP2P",
                    "nCompressP2L"):
            out[f"{name}_{key}"] = info[key]
        del S
    t0 = time.perf_counter()
    out["x_lu"] = K.dense_solve(B)
    print("dense LU", round(time.perf_counter() - t0, 1), "s", flush=True)
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "sphere7680_c3tol.npz")
    np.savez_compressed(path, **out)
    print("wrote", path)


if __name__ == "__main__":
    main(int(sys.argv[1]) if len(sys.argv) > 1 else (os.cpu_count() or 1))
