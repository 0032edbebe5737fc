"""Factorization checkpoint file (aifmm_solver_save / aifmm_solver_load): a
solver loaded from the file solves exactly as the solver that wrote it (same
blocks, same sweeps: bit-identical), for the plain path and for the mixed
factorization used as the FGMRES preconditioner; bad files and a kernel of
another size are rejected with an error status."""
import os

import numpy as np
import pytest

from rcs_b200 import mesh as M
from rcs_b200._lib import AifmmError
from rcs_b200.kernel import EFIEMatrix
from rcs_b200.solver import AIFMM, H2Operator

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def K():
    return EFIEMatrix(M.icosphere(3, 0.15), 1.0e9)


@pytest.mark.parametrize("precision", [0, 3])
def test_saved_factorization_solves_identically(K, tmp_path, precision):
    rng = np.random.default_rng(5)
    B = rng.standard_normal((K.N, 3)) + 1j * rng.standard_normal((K.N, 3))
    S = AIFMM(K, leaf_size=16, tol_pow=6, fillin_tol=8, n_levels=3, precision=precision)
    S.factorize()
    X1 = S.solve(B)
    path = str(tmp_path / "fac.bin")
    S.save(path)
    assert os.path.getsize(path) > 16 * K.N
    S2 = AIFMM.load(K, path)
    X2 = S2.solve(B)
    assert np.array_equal(X1, X2)
    i1, i2 = S.info(), S2.info()
    for key in ("n_levels", "start_level", "avg_leaf_size", "avg_multipoles", "max_rank"):
        assert i1[key] == i2[key], key
    if precision:
        A = H2Operator(K, leaf_size=16, tol_pow=10, n_levels=3)
        Xa, ra = S.solve_gmres(A, B, tol=1e-8)
        Xb, rb = S2.solve_gmres(A, B, tol=1e-8)
        assert ra["iterations"] == rb["iterations"] and np.array_equal(Xa, Xb)
        A.close()
    S.close()
    S2.close()


def test_bad_files_are_rejected(K, tmp_path):
    S = AIFMM(K, leaf_size=16, tol_pow=6, fillin_tol=8)
    with pytest.raises(AifmmError):
        S.save(str(tmp_path / "unfactored.bin"))  # nothing factorized yet
    S.factorize()
    path = str(tmp_path / "fac.bin")
    S.save(path)
    small = EFIEMatrix(M.icosphere(2, 0.15), 1.0e9)
    with pytest.raises(AifmmError):
        AIFMM.load(small, path)  # another unknown count
    junk = tmp_path / "junk.bin"
    junk.write_bytes(b"not a checkpoint" * 8)
    with pytest.raises(AifmmError):
        AIFMM.load(K, str(junk))
    data = open(path, "rb").read()
    cut = tmp_path / "cut.bin"
    cut.write_bytes(data[: len(data) // 2])
    with pytest.raises(AifmmError):
        AIFMM.load(K, str(cut))
    with pytest.raises(AifmmError):
        AIFMM.load(K, str(tmp_path / "missing.bin"))
    S.close()
