"""The CPU oracle against outputs of the reference itself (vaishna77/RCS
compiled from its unmodified sources; fixtures from
tests/golden/make_ref_golden.py): the pin of every parity claim that rests
on the oracle.

Bars: right-hand side and matrix entries bit-identical; the dense LU solution
to 1e-12; every box's rank after assembly and after factorization
identical; the AIFMM solution bit-identical where the factorization makes no
fill-in recompression (ACA 1e-8, RRQR 1e-10) and within 1e-7 (the RRQR
tolerance) where about 1,250 recompressions run (ACA 1e-5, RRQR 1e-7): the
oracle's norms and products round differently from the reference's build,
and a pivot of the column-pivoted QR or of ACA can then change between two
columns whose norms agree to rounding.  Every box's bases (L2P, P2M) agree
to 1e-12 after factorization and bit for bit after assembly; the leaf
level's bit for bit after factorization too wherever no recompression or a
third level is involved.  The L2M_f blocks, which the elimination factorizes
and inverts, carry the differences of the recompressions: to 1e-5 on two
levels, to 1e-3 on three, where the level-2 factors amplify the last-bit
differences of the basis updates and the solutions agree to 1.1e-6."""
import os

import numpy as np
import pytest

import oracle
from rcs_b200 import mesh as M

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = sorted(f[4:-4] for f in os.listdir(GOLDEN) if f.startswith("ref_") and f.endswith(".npz"))


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def bases(d):
    """The L2P, P2M and L2M_f rows of a block table (level, box, kind, key,
    rows, cols, norm)."""
    return d[np.isin(d[:, 2], (0, 1, 9))]


@pytest.fixture(scope="module", params=CASES)
def case(request):
    g = np.load(os.path.join(GOLDEN, f"ref_{request.param}.npz"))
    K = oracle.EFIE(M.Mesh(g["nodes"], g["tris"]), float(g["freq"]))
    return request.param, g, K


def test_fixtures_present():
    assert {"s78_l8_t8_f10", "s1280_l64_t8_f10", "s1280_l8_t5_f7", "s1280_l3_t5_f7"} <= set(CASES)


def test_rhs_and_entries(case):
    name, g, K = case
    assert K.N == int(g["N"])
    b = K.rhs_reference((1.0, 0.0, 0.0))
    assert np.array_equal(b, g["rhs"])
    ij = g["pairs"]
    rows, inv_r = np.unique(ij[:, 0], return_inverse=True)
    cols, inv_c = np.unique(ij[:, 1], return_inverse=True)
    A = K.matrix(rows.astype(np.int32), cols.astype(np.int32))
    assert np.array_equal(A[inv_r, inv_c], g["entries"])


def test_aifmm_solution_and_ranks(case):
    name, g, K = case
    b = np.asarray(g["rhs"])
    S = oracle.AIFMM(K, leaf_size=int(g["leaf"]), tol_pow=int(g["tol_pow"]), fillin_tol=int(g["fillin_tol"]))
    info = S.info()
    assert info["nLevels"] == int(g["nLevels"])
    d0 = S.dump()
    assert np.array_equal(d0[d0[:, 2] == 0][:, 5].astype(np.int32), g["rank_assembled"])
    # every box's assembled bases (L2P, P2M): same shapes, bit-identical norms
    assert np.array_equal(bases(d0), g["blocks_assembled"])
    S.factorize()
    x = S.solve(b)
    d1 = S.dump()
    assert np.array_equal(d1[d1[:, 2] == 0][:, 5].astype(np.int32), g["rank_factored"])
    f_o, f_r = bases(d1), g["blocks_factored"]
    assert np.array_equal(f_o[:, :6], f_r[:, :6])  # shapes of L2P, P2M, L2M_f after factorization
    leaf = f_r[:, 0] == int(g["nLevels"])
    scale = np.maximum(np.abs(f_r[:, 6]), 1e-300)
    if S.info()["nRRQR"] == 0 or int(g["nLevels"]) > 2:
        assert np.array_equal(f_o[leaf], f_r[leaf])  # leaf level: bit-identical
    rel_norm = np.abs(f_o[:, 6] - f_r[:, 6]) / scale
    assert np.max(rel_norm[f_r[:, 2] != 9]) < 1e-12  # L2P and P2M of every level
    # L2M_f carries the level-2 amplification on three levels (see the module docstring)
    assert np.max(rel_norm[f_r[:, 2] == 9]) < (1e-3 if int(g["nLevels"]) > 2 else 1e-5)
    if S.info()["nRRQR"] == 0:
        assert np.array_equal(x, g["x"])
    else:
        assert rel(x, g["x"]) < (1e-5 if int(g["nLevels"]) > 2 else 1e-7)
    if int(g["dense"]):
        assert rel(K.dense_solve(b), g["x_lu"]) < 1e-12
