"""GPU parity of the matrix-entry assembly kernels against the CPU oracle.

Bar: FP64 entries agree with the oracle to max|dZ| <= 1e-12 max|Z| (the two
use different exp/log/atan implementations; every other operation is the
same IEEE sequence); complex64 output within 1e-6 relative.
"""
import numpy as np
import pytest

import oracle
from rcs_b200 import mesh as M
from rcs_b200._lib import AifmmError
from rcs_b200.kernel import EFIEMatrix, ElectrostaticsMatrix

pytestmark = pytest.mark.gpu

GOLD = "tests/golden/sphere78.npz"


def rel_max(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLD)


def test_fixture78_dense_matches_golden(gold):
    m = M.Mesh(gold["nodes"], gold["tris"].astype(np.int32))
    K = EFIEMatrix(m, 1.0e7)
    assert K.N == 117
    A = K.dense()
    assert rel_max(A, gold["A"]) < 1e-12
    assert np.allclose(K.locations(), gold["locations"], rtol=0, atol=0)
    b = K.getRhs((1.0, 0.0, 0.0))
    assert rel_max(b, gold["rhs"]) < 1e-13


@pytest.mark.parametrize("sub,freq", [(3, 1.0e9), (4, 4.0e9)])
def test_efie_block_matches_oracle(sub, freq):
    m = M.icosphere(sub, 0.15)
    G = EFIEMatrix(m, freq)
    O = oracle.EFIE(m, freq)
    assert G.N == O.N
    rng = np.random.default_rng(sub)
    rows = rng.choice(G.N, size=min(G.N, 300), replace=False)
    cols = rng.choice(G.N, size=min(G.N, 257), replace=False)
    # include self and adjacent pairs (near zone, singular terms)
    cols[:40] = rows[:40]
    a = G.getMatrix(rows, cols)
    b = O.matrix(rows, cols)
    assert rel_max(a, b) < 1e-12
    big = np.abs(b) > 1e-6 * np.abs(b).max()
    assert np.max(np.abs(a - b)[big] / np.abs(b)[big]) < 1e-9


def test_efie_plane_projection_option():
    m = M.icosphere(3, 0.15)
    G = EFIEMatrix(m, 1.0e9)
    O = oracle.EFIE(m, 1.0e9)
    G.setPlaneProjection(True)
    O.set_plane_projection(True)
    idx = np.arange(0, G.N, 7)
    assert rel_max(G.getMatrix(idx, idx), O.matrix(idx, idx)) < 1e-12


def test_efie_complex64_output():
    m = M.icosphere(3, 0.15)
    G = EFIEMatrix(m, 1.0e9)
    idx = np.arange(0, G.N, 5)
    a64 = G.getMatrix(idx, idx, precision=1)
    a128 = G.getMatrix(idx, idx)
    assert a64.dtype == np.complex64
    assert rel_max(a64.astype(np.complex128), a128) < 1e-6


def test_rhs_matches_oracle():
    m = M.icosphere(3, 0.15)
    G = EFIEMatrix(m, 1.0e9)
    O = oracle.EFIE(m, 1.0e9)
    assert rel_max(G.getRhs(), O.rhs_reference()) < 1e-13
    e0 = np.array([1.0, 0.5j, 0.0])
    kh = np.array([0.0, 0.6, -0.8])
    assert rel_max(G.planeWaveRhs(kh, e0), O.rhs_plane(kh, e0)) < 1e-12


def test_electrostatics_matches_oracle():
    m = M.icosphere(3, 1.0)
    G = ElectrostaticsMatrix(m)
    O = oracle.Electrostatics(m)
    rng = np.random.default_rng(3)
    rows = rng.choice(G.N, 200, replace=False)
    cols = np.concatenate([rows[:50], rng.choice(G.N, 150, replace=False)])
    a = G.getMatrix(rows, cols)
    b = O.matrix(rows, cols)
    assert rel_max(a, b) < 1e-13
    assert np.all(a.imag == 0)
    assert np.array_equal(G.getRhs(1), np.ones(G.N))


def test_edge_cases():
    m = M.icosphere(2, 0.15)
    G = EFIEMatrix(m, 1.0e9)
    assert G.getMatrix([], [1, 2]).shape == (0, 2)
    with pytest.raises(AifmmError):
        G.getMatrix([G.N], [0])
    with pytest.raises(AifmmError):
        G.getMatrix([-1], [0])
    # a single row / column (kernel::getRow / getCol)
    r = G.getRow(3, np.arange(G.N))
    c = G.getCol(3, np.arange(G.N))
    A = G.dense()
    assert np.array_equal(r, A[3]) and np.array_equal(c, A[:, 3])
    # open surface: boundary edges are not unknowns (EFIEMatrix.cpp:199-209)
    half = M.Mesh(m.nodes, m.tris[: m.n_tris // 2].copy())
    Gh = EFIEMatrix(half, 1.0e9)
    assert Gh.N == M.rwg_count(half) == oracle.EFIE(half, 1.0e9).N
