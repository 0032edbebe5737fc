"""The GPU path against outputs of the reference itself (vaishna77/RCS built
from its unmodified sources; fixtures from tests/golden/make_ref_golden.py),
through the library's Python mirror of the reference classes.

Bars (plain complex128 path): right-hand side and seeded matrix entries to
1e-13 of their largest magnitude (the GPU's exp/sincos/log/atan differ from
the host's in the last bits); every box's rank after assembly and after
factorization identical to the reference's (every ACA, RRQR and queue
decision the same).  Solutions: the reference runs at its compiled-in 10 MHz,
where the 1,920-unknown sphere is electrically tiny (k a = 0.03) and its EFIE
matrix is ill-conditioned (the scalar-potential term dominates), so last-bit
differences of the entries move the solution by up to about 1e-6 even
without any recompression.  The bars are therefore the reference's own
accuracy: on the 117-unknown sphere the solution within 1e-10 of the
reference's; on the 1,920-unknown sphere the backward error ||Z x - b|| / ||b||
(Z assembled on the GPU) within twice the reference solution's, and the
solution itself within 1e-6 where no fill-in is recompressed, 1e-5 where it
is."""
import os

import numpy as np
import pytest

from rcs_b200 import mesh as M
from rcs_b200.kernel import EFIEMatrix
from rcs_b200.solver import AIFMM

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = ["s78_l8_t8_f10", "s1280_l64_t8_f10", "s1280_l8_t5_f7", "s1280_l3_t5_f7"]
SOLUTION_BAR = {"s78_l8_t8_f10": 1e-10, "s1280_l64_t8_f10": 1e-6, "s1280_l8_t5_f7": 1e-5, "s1280_l3_t5_f7": 1e-5}


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope="module", params=CASES)
def case(request):
    g = np.load(os.path.join(GOLDEN, f"ref_{request.param}.npz"))
    K = EFIEMatrix(M.Mesh(g["nodes"], g["tris"].astype(np.int32)), float(g["freq"]))
    return request.param, g, K


def test_rhs_and_entries(case):
    name, g, K = case
    assert K.N == int(g["N"])
    b = K.getRhs((1.0, 0.0, 0.0))
    assert np.max(np.abs(b - g["rhs"])) <= 1e-13 * np.max(np.abs(g["rhs"]))
    ij = g["pairs"]
    rows, inv_r = np.unique(ij[:, 0], return_inverse=True)
    cols, inv_c = np.unique(ij[:, 1], return_inverse=True)
    A = K.getMatrix(rows, cols)[inv_r, inv_c]
    assert np.max(np.abs(A - g["entries"])) <= 1e-13 * np.max(np.abs(g["entries"]))


@pytest.mark.parametrize("exact", [True, False])
def test_solution_and_ranks(case, exact):
    name, g, K = case
    S = AIFMM(K, leaf_size=int(g["leaf"]), tol_pow=int(g["tol_pow"]), fillin_tol=int(g["fillin_tol"]),
              exact_rrqr=exact)
    assert S.info()["n_levels"] == int(g["nLevels"])
    d0 = S.dump()
    assert np.array_equal(d0[d0[:, 2] == 0][:, 5].astype(np.int32), g["rank_assembled"])
    S.factorize()
    d1 = S.dump()
    assert np.array_equal(d1[d1[:, 2] == 0][:, 5].astype(np.int32), g["rank_factored"])
    x = S.solve(g["rhs"])
    assert rel(x, g["x"]) < SOLUTION_BAR[name], rel(x, g["x"])
    if K.N > 1000:  # backward error against the reference solution's, same dense matrix
        Z = K.getMatrix(np.arange(K.N), np.arange(K.N))
        b = np.asarray(g["rhs"])
        be = lambda y: float(np.linalg.norm(Z @ y - b) / np.linalg.norm(b))  # noqa: E731
        assert be(x) <= 2.0 * be(g["x"]) + 1e-14, (be(x), be(g["x"]))
    if int(g["dense"]):
        assert rel(x, g["x_lu"]) < 1e-5
    S.close()
