"""H^2 forward operator and FGMRES refinement against dense FP64 MoM.

The operator is checked against the dense EFIE/electrostatic matrix (entries
from the same kernel) on spheres small enough to hold densely; GMRES,
preconditioned by a loose factorization, must reach its residual target
measured with the DENSE matrix, not only with the operator it iterates on.
"""
import numpy as np
import pytest

from rcs_b200 import mesh as M
from rcs_b200.kernel import EFIEMatrix, ElectrostaticsMatrix
from rcs_b200.solver import AIFMM, H2Operator

pytestmark = pytest.mark.gpu


def _dense(K):
    idx = np.arange(K.N)
    return K.getMatrix(idx, idx)


def _rhs(N, nrhs, seed):
    rng = np.random.default_rng(seed)
    return rng.standard_normal((N, nrhs)) + 1j * rng.standard_normal((N, nrhs))


def _relerr(A, B):
    return float(np.linalg.norm(A - B) / np.linalg.norm(B))


@pytest.mark.parametrize("sub,freq,leaf,levels,tol_pow", [
    (3, 1.0e9, 64, 0, 10),    # 1,920 unknowns, the c1 sphere, the reference's depth rule
    (3, 4.0e9, 16, 3, 10),    # electrically larger, three levels
    (4, 2.0e9, 32, 3, 10),    # 7,680 unknowns
])
def test_operator_matches_dense(sub, freq, leaf, levels, tol_pow):
    K = EFIEMatrix(M.icosphere(sub, 0.15), freq)
    Z = _dense(K)
    A = H2Operator(K, leaf_size=leaf, tol_pow=tol_pow, n_levels=levels)
    X = _rhs(K.N, 3, 1)
    Y = A @ X
    err = _relerr(Y, Z @ X)
    assert err < 1e-7, err
    y0 = A @ X[:, 0]  # one column at a time gives the same product as the block
    assert np.allclose(y0, Y[:, 0], rtol=0, atol=1e-12 * np.abs(Y).max())


def test_operator_tolerance_controls_error():
    """The error falls with the ACA tolerance: the far field is in low-rank
    form (an all-dense operator would be exact at every tolerance)."""
    K = EFIEMatrix(M.icosphere(3, 0.15), 1.0e9)
    Z = _dense(K)
    X = _rhs(K.N, 2, 5)
    ops = [H2Operator(K, leaf_size=16, tol_pow=t, n_levels=3) for t in (4, 7, 10)]
    errs = [_relerr(A @ X, Z @ X) for A in ops]
    assert errs[0] > errs[1] > errs[2], errs
    assert errs[2] < 1e-7, errs


def test_operator_column_chunks():
    """More columns than one skinny pass takes (16) go through in chunks."""
    K = EFIEMatrix(M.icosphere(2, 0.15), 1.0e9)
    Z = _dense(K)
    A = H2Operator(K, leaf_size=8, tol_pow=10, n_levels=3)
    X = _rhs(K.N, 19, 2)
    assert _relerr(A @ X, Z @ X) < 1e-7


def test_operator_electrostatics():
    K = ElectrostaticsMatrix(M.icosphere(3, 1.0))
    Z = _dense(K)
    X = _rhs(K.N, 2, 3)
    loose = _relerr(H2Operator(K, leaf_size=16, tol_pow=4, n_levels=3) @ X, Z @ X)
    tight = _relerr(H2Operator(K, leaf_size=16, tol_pow=10, n_levels=3) @ X, Z @ X)
    assert tight < 1e-7 and loose > 10 * tight, (loose, tight)


@pytest.mark.parametrize("tol", [1e-6, 1e-8])
def test_gmres_reaches_dense_residual(tol):
    """Loose factorization (ACA 1e-4) + tight operator (1e-11): the true residual
    ||Z x - b|| / ||b|| with the dense matrix meets the target."""
    K = EFIEMatrix(M.icosphere(3, 0.15), 1.0e9)
    Z = _dense(K)
    S = AIFMM(K, leaf_size=16, tol_pow=4, fillin_tol=6, n_levels=3)
    S.factorize()
    A = H2Operator(K, leaf_size=16, tol_pow=11, n_levels=3)
    B = np.stack([K.planeWaveRhs((0, 0, -1), (1, 0, 0)), K.planeWaveRhs((1, 0, 0), (0, 1, 0)),
                  _rhs(K.N, 1, 4)[:, 0]], axis=1)
    direct_res = np.linalg.norm(Z @ S.solve(B) - B) / np.linalg.norm(B)
    X, rec = S.solve_gmres(A, B, tol=tol, restart=30, maxit=100)
    true_res = max(np.linalg.norm(Z @ X[:, c] - B[:, c]) / np.linalg.norm(B[:, c]) for c in range(B.shape[1]))
    assert rec["relres"] <= tol
    assert true_res <= 2 * tol, (true_res, rec, direct_res)
    assert rec["iterations"] >= 1
    assert direct_res > tol  # the refinement did the work


def test_gmres_zero_rhs_and_bad_arguments():
    from rcs_b200._lib import AifmmError
    K = EFIEMatrix(M.icosphere(2, 0.15), 1.0e9)
    S = AIFMM(K, leaf_size=16, tol_pow=6, fillin_tol=8)
    S.factorize()
    A = H2Operator(K, leaf_size=16, tol_pow=10)
    X, rec = S.solve_gmres(A, np.zeros(K.N, dtype=np.complex128))
    assert np.all(X == 0) and rec["iterations"] == 0
    with pytest.raises(AifmmError):
        S.solve_gmres(A, np.ones(K.N), tol=-1.0)
    K2 = EFIEMatrix(M.icosphere(3, 0.15), 1.0e9)
    A2 = H2Operator(K2, leaf_size=64, tol_pow=8)
    with pytest.raises(AifmmError):  # sizes differ
        S.solve_gmres(A2, np.ones(K.N))


def test_mixed_precision_factorization_refines_to_target():
    """precision=1 (split-TF32 tensor-core elimination GEMMs) as the
    preconditioner: GMRES reaches 1e-8 against the dense matrix, and the
    mixed direct solve is no worse than FP32-level noise on top of the plain one."""
    K = EFIEMatrix(M.icosphere(3, 0.15), 1.0e9)
    Z = _dense(K)
    b = K.planeWaveRhs((0, 0, -1), (1, 0, 0))
    A = H2Operator(K, leaf_size=16, tol_pow=11, n_levels=3)
    res = {}
    for prec in (0, 1, 3):
        S = AIFMM(K, leaf_size=16, tol_pow=6, fillin_tol=8, n_levels=3, precision=prec)
        S.factorize()
        res[prec] = np.linalg.norm(Z @ S.solve(b) - b) / np.linalg.norm(b)
        x, rec = S.solve_gmres(A, b, tol=1e-8)
        assert np.linalg.norm(Z @ x - b) / np.linalg.norm(b) < 2e-8, (prec, rec)
    assert res[1] < max(10 * res[0], 1e-5) and res[3] < max(10 * res[0], 1e-5), res
