"""Solve sweeps replayed from a captured CUDA graph: the same kernels with the
same arguments as the sweep issued launch by launch, so the solutions are
bit-identical; one capture per factorization and right-hand-side count, and
a refactorization or a rewind captures again (its blocks moved)."""
import numpy as np
import pytest

from rcs_b200 import mesh as M
from rcs_b200.kernel import EFIEMatrix
from rcs_b200.solver import AIFMM, H2Operator, launch_count

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def K():
    return EFIEMatrix(M.icosphere(3, 0.15), 1.0e9)


def _rhs(n, nrhs, seed):
    rng = np.random.default_rng(seed)
    return rng.standard_normal((n, nrhs)) + 1j * rng.standard_normal((n, nrhs))


@pytest.mark.parametrize("precision", [0, 3])
def test_graph_solve_matches_launch_by_launch(K, precision):
    B3, B1 = _rhs(K.N, 3, 1), _rhs(K.N, 1, 2)
    S = AIFMM(K, leaf_size=16, tol_pow=6, fillin_tol=8, n_levels=3, precision=precision)
    S.checkpoint()
    S.factorize()
    S.set_graph_solve(False)
    E3, E1 = S.solve(B3), S.solve(B1)
    assert S.info()["n_solve_graph"] == 0
    S.set_graph_solve(True)
    l0 = launch_count()
    G3 = S.solve(B3)  # captures, then replays
    l1 = launch_count()
    G3b = S.solve(B3)  # replays
    l2 = launch_count()
    G1 = S.solve(B1)  # another right-hand-side count: captures again
    info = S.info()
    assert info["n_solve_capture"] == 2 and info["n_solve_graph"] == 3
    assert np.array_equal(G3, E3) and np.array_equal(G3b, E3) and np.array_equal(G1, E1)
    # a replay counts the graph's kernels, the capture itself launches nothing
    assert l2 - l1 == l1 - l0 > 50
    # a refactorization drops the plan: the next solve captures the new blocks
    S.rewind()
    S.factorize()
    G3c = S.solve(B3)
    assert S.info()["n_solve_capture"] == 3
    S.set_graph_solve(False)
    E3c = S.solve(B3)
    assert np.array_equal(G3c, E3c)
    # the refactorization starts from a copy of the assembled blocks, and the
    # first factorization after assembly rounds differently (about 1e-15);
    # split TF32 amplifies that to FP32-level differences
    assert np.linalg.norm(G3c - E3) <= (1e-8 if precision == 0 else 1e-4) * np.linalg.norm(E3)
    S.close()


def test_graph_solve_inside_fgmres(K):
    B = _rhs(K.N, 2, 3)
    A = H2Operator(K, leaf_size=16, tol_pow=10, n_levels=3)
    runs = []
    for on in (False, True):
        S = AIFMM(K, leaf_size=16, tol_pow=6, fillin_tol=8, n_levels=3, precision=3, drop_pow=2)
        S.set_graph_solve(on)
        S.factorize()
        X, r = S.solve_gmres(A, B, tol=1e-8)
        runs.append((X, r["iterations"], S.info()["n_solve_graph"]))
        S.close()
    A.close()
    (Xe, ie, ge), (Xg, ig, gg) = runs
    assert ge == 0 and gg == ig  # one preconditioner application per iteration, each replayed
    assert ie == ig and np.array_equal(Xe, Xg)
