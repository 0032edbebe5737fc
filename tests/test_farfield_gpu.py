"""Far field on the GPU: centroid currents and the one-point RCS
(EFIEMatrix::getJAtCentroids, src/EFIEMatrix.cpp:1100-1130, and
getRCS_OnePointQuadrature, :916-930) against their restatement in
tests/physics.py (currents to 1e-12, RCS to 1e-10 relative: the GPU sums the
triangles in a different order), and the AIFMM-solved RCS of a PEC sphere
against the Mie series (within 1 dB, as the oracle's own pin).  Also the
solver built over caller-given locations and its tree order."""
import numpy as np
import pytest

from rcs_b200 import mesh as M
from rcs_b200.kernel import EFIEMatrix
from rcs_b200.solver import AIFMM
from tests import physics

import oracle

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def sphere():
    m = M.icosphere(3, 0.15)
    K = EFIEMatrix(m, 1.0e9)
    O = oracle.EFIE(m, 1.0e9)
    rwg, ln = O.rwg()
    return m, K, rwg, ln


def test_currents_and_rcs_match_restatement(sphere):
    m, K, rwg, ln = sphere
    rng = np.random.default_rng(11)
    x = rng.standard_normal(K.N) + 1j * rng.standard_normal(K.N)
    J = K.getJAtCentroids(x)
    Jr, cen, area = physics.centroid_currents(m, rwg, ln, x)
    assert J.shape == (m.n_tris, 3) and _rel(J, Jr) < 1e-12
    k = 2 * np.pi * 1.0e9 / 3.0e8
    for phi in (0.0, 0.7):
        th = np.linspace(0, np.pi, 37)
        got = K.getRCS_OnePointQuadrature(th, phi, J)
        ref = physics.rcs_one_point(Jr, cen, area, k, th, phi)
        assert np.allclose(got, ref, rtol=1e-10, atol=1e-12 * ref.max())
    one = K.getRCS_OnePointQuadrature(0.3, 0.2, J)  # scalar angle
    assert one.shape == (1,) and np.isclose(one[0], physics.rcs_one_point(Jr, cen, area, k, [0.3], 0.2)[0],
                                            rtol=1e-10)


def test_rcs_of_solved_sphere_follows_mie(sphere):
    m, _, rwg, ln = sphere
    K = EFIEMatrix(m, 1.0e9)
    K.setPlaneProjection(True)
    S = AIFMM(K, leaf_size=64, tol_pow=10, fillin_tol=12)
    S.factorize()
    x = S.solve(K.planeWaveRhs((0, 0, -1), (1, 0, 0)))
    J = K.getJAtCentroids(x)
    k = 2 * np.pi * 1.0e9 / 3.0e8
    th = np.linspace(0, np.pi, 19)
    num = 10 * np.log10(K.getRCS_OnePointQuadrature(th, 0.0, J))
    mie = 10 * np.log10(physics.mie_pec_rcs(k * 0.15, k, np.pi - th, 0.0))
    assert np.max(np.abs(num - mie)) < 1.0


def test_solver_over_given_locations_and_tree_order(sphere):
    _, K, _, _ = sphere
    b = K.getRhs()
    S0 = AIFMM(K, leaf_size=64, tol_pow=8, fillin_tol=10)
    S0.factorize()
    x0 = S0.solve(b)
    loc = K.locations()
    lo, hi = loc.min(axis=0), loc.max(axis=0)
    dom = np.array([lo[0], hi[0], lo[1], hi[1], lo[2], hi[2]])
    S1 = AIFMM(K, leaf_size=64, tol_pow=8, fillin_tol=10, locations=loc, domain=dom)
    S1.factorize()
    assert _rel(S1.solve(b), x0) < 1e-13  # same locations and box: the same solver
    order = S1.tree_order()
    assert sorted(order.tolist()) == list(range(K.N))
    # a wider box changes the octree, not the answer beyond the tolerances
    S2 = AIFMM(K, leaf_size=64, tol_pow=8, fillin_tol=10, locations=loc, domain=dom * 1.5)
    S2.factorize()
    assert _rel(S2.solve(b), x0) < 1e-5
    from rcs_b200._lib import AifmmError
    with pytest.raises(AifmmError):  # the box must contain every location
        AIFMM(K, leaf_size=64, locations=loc, domain=dom * 0.5)
