"""Batched bodies (aifmm_batch_factorize / aifmm_batch_solve_gmres): each
body of a concurrent batch gets exactly the factorization and the solution
that the one-body calls give it; a batch that shares a context is refused."""
import numpy as np
import pytest

from rcs_b200 import batch
from rcs_b200._lib import AifmmError
from rcs_b200.kernel import Context, EFIEMatrix
from rcs_b200.solver import AIFMM, H2Operator

pytestmark = pytest.mark.gpu


def _bodies(n, precision):
    out = []
    for mesh, axes in batch.ellipsoid_family(n, seed=64, subdivisions=(2, 3)):
        ctx = Context(0)
        K = EFIEMatrix(mesh, 2.0e9, ctx=ctx)
        S = AIFMM(K, leaf_size=16, tol_pow=5, fillin_tol=7, n_levels=3, precision=precision)
        out.append((ctx, K, S))
    return out


@pytest.mark.parametrize("precision", [0, 4])
def test_batch_equals_one_by_one(precision):
    bodies = _bodies(6, precision)
    rng = np.random.default_rng(3)
    rhs = [rng.standard_normal((K.N, 2)) + 1j * rng.standard_normal((K.N, 2)) for _, K, _ in bodies]
    for _, _, S in bodies:
        S.checkpoint()
    for _, _, S in bodies:  # one by one, from the checkpoint (the batch's starting point)
        S.rewind()
        S.factorize()
    single = [S.solve(b) for (_, _, S), b in zip(bodies, rhs)]
    for _, _, S in bodies:
        S.rewind()
    sec = batch.batch_factorize([S for _, _, S in bodies], threads=4)
    assert sec > 0
    for (_, _, S), b, x in zip(bodies, rhs, single):
        assert np.array_equal(S.solve(b), x)
    ops = [H2Operator(K, leaf_size=16, tol_pow=10, n_levels=3) for _, K, _ in bodies]
    xs, recs, _ = batch.batch_solve_gmres([S for _, _, S in bodies], ops, rhs, tol=1e-8, threads=4)
    for (_, K, S), A, b, x, r in zip(bodies, ops, rhs, xs, recs):
        x1, r1 = S.solve_gmres(A, b, tol=1e-8)
        assert r["iterations"] == r1["iterations"] and np.array_equal(x, x1)
        assert r["relres"] <= 1e-8


def test_batch_needs_one_context_per_body():
    ctx = Context(0)
    Ks = [EFIEMatrix(m, 2.0e9, ctx=ctx) for m, _ in batch.ellipsoid_family(2, subdivisions=(2,))]
    Ss = [AIFMM(K, leaf_size=16, tol_pow=5, fillin_tol=7) for K in Ks]
    with pytest.raises(AifmmError):
        batch.batch_factorize(Ss)
