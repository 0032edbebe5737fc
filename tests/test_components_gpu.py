"""GPU low-rank / dense components against the CPU oracle.

ACA: identical pivots and rank (integer parity), original rows/columns to
1e-12 relative.  RRQR: identical rank, Q_trunc spanning the same space and
equal up to the rounding of a Householder QR (1e-10), maxPivot to 1e-12.
LU solve: residual at rounding level.
"""
import numpy as np
import pytest

import oracle
from rcs_b200 import lowrank
from rcs_b200 import mesh as M
from rcs_b200.kernel import EFIEMatrix

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("zsplit,tol", [(0.11, 1e-8), (0.05, 1e-5), (0.0, 1e-10)])
def test_aca_matches_oracle(zsplit, tol):
    m = M.icosphere(3, 0.15)
    K = EFIEMatrix(m, 1.0e9)
    O = oracle.EFIE(m, 1.0e9)
    loc = K.locations()
    rows = np.where(loc[:, 2] > zsplit)[0]
    cols = np.where(loc[:, 2] < -zsplit)[0][:150]
    for r_, c_ in ((rows, cols), (cols, rows)):  # both branches of ACA_only_nodes2
        rb, cb, Ac, Ar = lowrank.ACA_only_nodes2(K, r_, c_, tol)
        orb, ocb, oAc, oAr = oracle.aca(O, r_, c_, tol)
        assert np.array_equal(rb, orb) and np.array_equal(cb, ocb)
        assert rel(Ac, oAc) < 1e-12 and rel(Ar, oAr) < 1e-12


def _rrqr_case(seed, m, r0, nf, frank):
    rng = np.random.default_rng(seed)
    U = rng.standard_normal((m, r0)) + 1j * rng.standard_normal((m, r0))
    U *= np.logspace(0, -12, r0)[None, :]  # graded old basis: partition-1 truncation fires
    F = (rng.standard_normal((m, frank)) + 1j * rng.standard_normal((m, frank))) @ \
        (rng.standard_normal((frank, nf)) + 1j * rng.standard_normal((frank, nf)))
    return np.hstack([U, F])


@pytest.mark.parametrize("seed,m,r0,nf,frank,tp1,tp2,fr,ip", [
    (1, 40, 6, 12, 3, 10, 10, 5, 1.0),
    (2, 60, 10, 30, 8, 8, 10, 5, 10.0),     # partition-1 early exit + fill-in cap
    (3, 25, 12, 40, 20, 6, 8, 10, 0.5),     # more columns than rows
    (4, 50, 0, 20, 7, 8, 9, 10, 2.0),       # no old basis
])
def test_rrqr_matches_oracle(seed, m, r0, nf, frank, tp1, tp2, fr, ip):
    A = _rrqr_case(seed, m, r0, nf, frank)
    Q, mp = lowrank.RRQR(A, tp1, tp2, r0, ip, fr)
    Qo, Ro, perm, mpo, err = oracle.rrqr(A, tp1, tp2, r0, ip, fr)
    assert Q.shape == Qo.shape
    assert abs(mp - mpo) <= 1e-12 * max(mpo, 1.0)
    if Q.shape[1]:
        assert np.allclose(Q.conj().T @ Q, np.eye(Q.shape[1]), atol=1e-12)
        assert rel(Q, Qo) < 1e-10


def test_lu_solve():
    rng = np.random.default_rng(0)
    for n in (1, 31, 32, 33, 200, 517):
        A = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
        B = rng.standard_normal((n, 3)) + 1j * rng.standard_normal((n, 3))
        X = lowrank.lu_solve(A, B)
        assert np.linalg.norm(A @ X - B) / np.linalg.norm(B) < 1e-11
