"""GPU AIFMM (plain complex128 path) against the CPU oracle.

The plain FP64 GPU path follows the reference's control flow (same tree,
same ACA pivots, same queues and elimination order), so its solution must
match the oracle's AIFMM solution to 1e-10 relative, and its structural
statistics (ranks, numbers of recompressions) must be identical.
"""
import numpy as np
import pytest

import oracle
from rcs_b200 import mesh as M
from rcs_b200.kernel import EFIEMatrix, ElectrostaticsMatrix
from rcs_b200.solver import AIFMM

pytestmark = pytest.mark.gpu

PARITY = 1e-10


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_fixture78_matches_oracle_solution():
    g = np.load("tests/golden/sphere78.npz")
    m = M.Mesh(g["nodes"], g["tris"].astype(np.int32))
    K = EFIEMatrix(m, 1.0e7)
    S = AIFMM(K, leaf_size=8, tol_pow=8, fillin_tol=10)
    S.factorize()
    x = S.solve(g["rhs"])
    assert rel(x, g["x_aifmm"]) < PARITY
    assert rel(x, g["x_lu"]) < 1e-9
    A = g["A"]
    assert np.linalg.norm(A @ x - g["rhs"]) / np.linalg.norm(g["rhs"]) < 1e-10


@pytest.mark.parametrize("exact", [True, False])
@pytest.mark.parametrize("sub,freq,leaf,tol,ftol,nl", [
    (3, 1.0e9, 64, 8, 10, 0),   # config 1 with the reference's depth rule (2 levels)
    (3, 1.0e9, 16, 6, 8, 3),    # three levels: RRQR recompression and a non-leaf level
    (3, 4.0e9, 8, 5, 7, 3),     # loose tolerances, many recompressions of orthonormal bases
])
def test_sphere_matches_oracle(sub, freq, leaf, tol, ftol, nl, exact):
    """exact=True runs every RRQR through the reference's full partition-1
    pass; exact=False keeps orthonormal old bases (same ranks and spans)."""
    m = M.icosphere(sub, 0.15)
    K = EFIEMatrix(m, freq)
    O = oracle.EFIE(m, freq)
    b = K.planeWaveRhs((0, 0, -1), (1, 0, 0))
    S = AIFMM(K, leaf_size=leaf, tol_pow=tol, fillin_tol=ftol, n_levels=nl, exact_rrqr=exact)
    S.factorize()
    x = S.solve(b)
    SO = oracle.AIFMM(O, leaf_size=leaf, tol_pow=tol, fillin_tol=ftol, n_levels=nl)
    SO.factorize()
    xo = SO.solve(b)
    gi, oi = S.info(), SO.info()
    assert gi["n_levels"] == oi["nLevels"] and gi["start_level"] == oi["startLevel"]
    assert gi["avg_leaf_size"] == oi["avgLeafSize"]
    assert gi["max_rank"] == oi["maxRank"]
    assert gi["n_rrqr"] == oi["nRRQR"]
    assert gi["n_compress_p2p"] == oi["nCompressP2P"] and gi["n_compress_p2l"] == oi["nCompressP2L"]
    assert rel(x, xo) < PARITY


def test_multiple_rhs_equal_single_solves():
    m = M.icosphere(3, 0.15)
    K = EFIEMatrix(m, 1.0e9)
    S = AIFMM(K, leaf_size=64, tol_pow=8, fillin_tol=10)
    S.factorize()
    B = np.stack([K.planeWaveRhs((0, 0, -1), (1, 0, 0)), K.planeWaveRhs((1, 0, 0), (0, 1j, 0)),
                  K.getRhs((1.0, 0.0, 0.0))], axis=1)
    X = S.solve(B)
    for c in range(B.shape[1]):
        assert rel(X[:, c], S.solve(B[:, c])) < 1e-13


@pytest.mark.parametrize("exact,nl", [(True, 0), (False, 0), (False, 3)])
def test_electrostatics_capacitance(exact, nl):
    m = M.icosphere(3, 1.0)
    K = ElectrostaticsMatrix(m)
    O = oracle.Electrostatics(m)
    S = AIFMM(K, leaf_size=16, tol_pow=8, fillin_tol=10, n_levels=nl, exact_rrqr=exact)
    S.factorize()
    sigma = S.solve(np.ones(K.N))
    SO = oracle.AIFMM(O, leaf_size=16, tol_pow=8, fillin_tol=10, n_levels=nl)
    SO.factorize()
    so = SO.solve(np.ones(K.N))
    assert rel(sigma, so) < PARITY
    v = m.nodes[m.tris - 1]
    area = 0.5 * np.linalg.norm(np.cross(v[:, 1] - v[:, 0], v[:, 2] - v[:, 0]), axis=1)
    C = float(np.real(sigma) @ area)
    assert abs(C / (4 * np.pi * 8.854187817e-12) - 1) < 0.02


def test_solve_before_factorize_is_an_error():
    from rcs_b200._lib import AifmmError
    m = M.icosphere(2, 0.15)
    K = EFIEMatrix(m, 1.0e9)
    S = AIFMM(K, leaf_size=16, tol_pow=8, fillin_tol=10)
    with pytest.raises(AifmmError):
        S.solve(np.ones(K.N))
