"""Plain and mixed GPU paths against the CPU oracle at the benchmark's
tolerances (ACA 1e-5, RRQR 1e-7, f = 4 GHz, R = 0.15 m) on the 7,680-unknown
sphere, for two tree shapes: the reference's depth rule at leaf size 128
(one level of 56 boxes of about 137 unknowns) and the benchmark's depth of
three levels.  The oracle's outputs come from tests/golden/make_c3tol.py
(the oracle needs minutes at this size).

Bars: the plain FP64 path reproduces the reference algorithm -- identical
tree statistics, ranks and recompression counts with either RRQR mode, and
the solution within 1e-10 of the oracle's AIFMM solution on the two-level
tree.  On the three-level tree the non-leaf elimination amplifies rounding:
the reference itself, built from its own sources, and the oracle agree
bit for bit on every leaf-level block after factorization and to 1e-15 on the
level-2 bases, yet their solutions differ by 1.1e-6 (three levels, 1,920
unknowns, the same tolerances; tests/golden/ref_s1280_l3_t5_f7.npz), because
the level-2 LU factors and inverses magnify the last-bit differences of the
basis updates.  The bar there is therefore the integer decisions (ranks,
counts) plus the ACA tolerance, 1e-5, on the solution.  The mixed path
(split-TF32 tensor-core Schur products) refined by FP64 FGMRES reaches the
dense FP64 solution to 1e-6 relative."""
import os

import numpy as np
import pytest

from rcs_b200 import mesh as M
from rcs_b200.kernel import EFIEMatrix
from rcs_b200.solver import AIFMM, H2Operator

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "sphere7680_c3tol.npz")
PARITY = {"leaf128": 1e-10, "lvl3": 1e-5}


@pytest.fixture(scope="module")
def fx():
    g = np.load(GOLDEN)
    K = EFIEMatrix(M.icosphere(int(g["sub"]), float(g["radius"])), float(g["freq"]))
    return g, K


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("exact", [True, False])
@pytest.mark.parametrize("shape", ["leaf128", "lvl3"])
def test_plain_matches_oracle(fx, shape, exact):
    g, K = fx
    S = AIFMM(K, leaf_size=int(g[f"{shape}_leaf"]), tol_pow=int(g["tol_pow"]), fillin_tol=int(g["fillin_tol"]),
              n_levels=int(g[f"{shape}_levels"]), exact_rrqr=exact)
    S.factorize()
    X = S.solve(g["rhs"])
    i = S.info()
    assert i["n_levels"] == g[f"{shape}_nLevels"] and i["start_level"] == g[f"{shape}_startLevel"]
    assert i["avg_leaf_size"] == g[f"{shape}_avgLeafSize"]
    assert i["avg_multipoles"] == g[f"{shape}_avgMultipoles"] and i["max_rank"] == g[f"{shape}_maxRank"]
    assert i["n_rrqr"] == g[f"{shape}_nRRQR"]
    assert i["n_compress_p2p"] == g[f"{shape}_nCompressP2P"] and i["n_compress_p2l"] == g[f"{shape}_nCompressP2L"]
    for c in range(X.shape[1]):
        assert rel(X[:, c], g[f"{shape}_x"][:, c]) < PARITY[shape]
    S.close()


def test_rhs_matches_oracle(fx):
    import bench
    g, K = fx
    B = np.stack([K.planeWaveRhs(k, e) for k, e in bench.plane_waves(2)], axis=1)
    assert rel(B, g["rhs"]) < 1e-14


@pytest.mark.parametrize("shape", ["leaf128", "lvl3"])
def test_mixed_refined_reaches_dense_solution(fx, shape):
    """The mixed factorization is a preconditioner: after FGMRES to 1e-10 on
    a tight forward operator, the solution agrees with the oracle's dense LU
    solution to 1e-6 (the oracle's AIFMM solution itself is only an ACA-1e-5
    approximation and differs from both by more)."""
    g, K = fx
    lv = int(g[f"{shape}_levels"])
    S = AIFMM(K, leaf_size=int(g[f"{shape}_leaf"]), tol_pow=int(g["tol_pow"]), fillin_tol=int(g["fillin_tol"]),
              n_levels=lv, precision=3)
    S.factorize()
    A = H2Operator(K, leaf_size=int(g[f"{shape}_leaf"]), tol_pow=12, n_levels=lv)
    X, rec = S.solve_gmres(A, g["rhs"], tol=1e-10, restart=30, maxit=200)
    for c in range(X.shape[1]):
        assert rel(X[:, c], g["x_lu"][:, c]) < 1e-6, (c, rel(X[:, c], g["x_lu"][:, c]), rec)
    # the oracle's AIFMM solution (ACA 1e-5) is farther from the dense one
    assert rel(g[f"{shape}_x"][:, 0], g["x_lu"][:, 0]) > rel(X[:, 0], g["x_lu"][:, 0])
    S.close()
    A.close()


def test_mixed_refined_matches_oracle_aifmm_at_config1():
    """At the reference's own tight tolerances (config 1: N = 1,920, leaf 64,
    ACA 1e-8, RRQR 1e-10, f = 1 GHz) the oracle's AIFMM solve is accurate to
    about 1e-8, and the mixed factorization refined by FGMRES matches it to
    1e-6 (the stated bar for the mixed form)."""
    import oracle
    m = M.icosphere(3, 0.15)
    K = EFIEMatrix(m, 1.0e9)
    O = oracle.EFIE(m, 1.0e9)
    b = K.planeWaveRhs((0, 0, -1), (1, 0, 0))
    SO = oracle.AIFMM(O, leaf_size=64, tol_pow=8, fillin_tol=10)
    SO.factorize()
    xo = SO.solve(b)
    S = AIFMM(K, leaf_size=64, tol_pow=8, fillin_tol=10, precision=3)
    S.factorize()
    A = H2Operator(K, leaf_size=64, tol_pow=12)
    x, rec = S.solve_gmres(A, b, tol=1e-10)
    assert rel(x, xo) < 1e-6, (rel(x, xo), rec)
