"""The electrostatics configuration (c2) at a small size: a mixed
factorization of the unit-sphere collocation system (split-TF32 tensor-core
Schur products with FP32 accumulation: FP32-class accuracy) used as the
preconditioner of FP64 FGMRES to a relative residual of 1e-8, with 32 seeded
N(0,1) potential right-hand sides plus the 1 V conductor right-hand side
(ElectrostaticsMatrix::getRhs, src/ElectrostaticsMatrix.cpp:374-381).  Checked
against the dense matrix (residual), the CPU oracle's dense solve (the 1 V
charge density) and the analytic capacitance 4 pi eps0 R
(getCapacitance, :366-402)."""
import numpy as np
import pytest

import oracle
from rcs_b200 import mesh as M
from rcs_b200.kernel import ElectrostaticsMatrix
from rcs_b200.solver import AIFMM, H2Operator

pytestmark = pytest.mark.gpu

EPS0 = 8.854187817e-12


def es_rhs(K, n_random: int, seed: int = 20261203) -> np.ndarray:
    """n_random seeded N(0,1) potential vectors (one per column) and the 1 V
    conductor right-hand side last."""
    rng = np.random.Generator(np.random.MT19937(seed))
    R = rng.standard_normal((K.N, n_random))
    return np.concatenate([R, K.getRhs(1)[:, None]], axis=1).astype(np.complex128)


def test_c2_mixed_factorization_refines_to_1e8():
    m = M.icosphere(4, 1.0)
    K = ElectrostaticsMatrix(m)
    B = es_rhs(K, 32)
    S = AIFMM(K, leaf_size=32, tol_pow=5, fillin_tol=7, n_levels=3, precision=3)
    S.factorize()
    A = H2Operator(K, leaf_size=32, tol_pow=11, n_levels=3)
    X, rec = S.solve_gmres(A, B, tol=1e-8, restart=30, maxit=100)
    idx = np.arange(K.N)
    Z = K.getMatrix(idx, idx)
    res = np.linalg.norm(Z @ X - B, axis=0) / np.linalg.norm(B, axis=0)
    assert res.max() <= 2e-8, (res.max(), rec)
    assert np.abs(X.imag).max() <= 1e-12 * np.abs(X.real).max()  # a real system stays real
    # the direct solve with the FP32-class factorization alone is far from 1e-8
    direct = np.linalg.norm(Z @ S.solve(B[:, -1]) - B[:, -1]) / np.linalg.norm(B[:, -1])
    assert direct > 1e-8
    # 1 V solution against the oracle's dense LU (src/ElectrostaticsMatrix.cpp:342-364)
    O = oracle.Electrostatics(m)
    so = O.dense_solve(B[:, -1])
    sigma = X[:, -1]
    assert np.linalg.norm(sigma - so) / np.linalg.norm(so) < 1e-6
    v = m.nodes[m.tris - 1]
    area = 0.5 * np.linalg.norm(np.cross(v[:, 1] - v[:, 0], v[:, 2] - v[:, 0]), axis=1)
    C = float(np.real(sigma) @ area)
    assert abs(C / (4 * np.pi * EPS0 * 1.0) - 1) < 0.02
