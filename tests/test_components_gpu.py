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


def _single_kernel_rrqr(A, tp1, tp2, part, pivot, fill):
    """The one-CTA RRQR kernel, reached through the allocation-free entry point."""
    import ctypes as C
    import torch
    from rcs_b200 import _lib
    m, n = A.shape
    Ad = torch.from_numpy(np.ascontiguousarray(A.T)).cuda()
    Qd = torch.zeros((min(m, n) + 1, m), dtype=torch.complex128, device="cuda")
    rk = torch.zeros(1, dtype=torch.int32, device="cuda")
    mp = torch.zeros(1, dtype=torch.float64, device="cuda")
    _lib.check(_lib.lib().aifmm_rrqr_noalloc(C.c_void_p(Ad.data_ptr()), m, n, part, tp1, tp2, float(pivot), fill, 0,
                                             C.c_void_p(Qd.data_ptr()), C.c_void_p(rk.data_ptr()),
                                             C.c_void_p(mp.data_ptr()), None))
    torch.cuda.synchronize()
    r = int(rk.item())
    return Qd.cpu().numpy()[:r].T, float(mp.item())


@pytest.mark.parametrize("seed,m,r0,nf,frank,tp1,tp2,fr,ip", [
    (2, 60, 10, 30, 8, 8, 10, 5, 10.0),
    (3, 25, 12, 40, 20, 6, 8, 10, 0.5),
    (4, 50, 0, 20, 7, 8, 9, 10, 2.0),
    (5, 300, 90, 1200, 60, 7, 9, 10, 1.0),   # fill-in recompression shape of a 128-unknown leaf level
    (6, 200, 200, 0, 1, 7, 9, 5, 1.0),       # no fill-in columns
])
def test_rrqr_split_pipeline_bit_exact(seed, m, r0, nf, frank, tp1, tp2, fr, ip):
    """The four-launch RRQR used by the solver equals the one-CTA kernel bit for bit."""
    A = _rrqr_case(seed, m, r0, nf, frank) if nf else _rrqr_case(seed, m, r0, 1, 1)[:, :r0]
    Q1, mp1 = _single_kernel_rrqr(A, tp1, tp2, r0, ip, fr)
    Q4, mp4 = lowrank.RRQR(A, tp1, tp2, r0, ip, fr)
    assert Q1.shape == Q4.shape and mp1 == mp4
    assert np.array_equal(Q1, Q4)


@pytest.mark.parametrize("nrhs", [1, 3, 16, 17])
def test_lu_solve(nrhs):
    # 16 columns x 700 rows is the largest case of the one-CTA shared-memory
    # solve here; 800 x 16 and 17 columns take the blocked path.
    rng = np.random.default_rng(nrhs)
    for n in (1, 31, 32, 33, 200, 517, 700, 800):
        A = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
        B = rng.standard_normal((n, nrhs)) + 1j * rng.standard_normal((n, nrhs))
        X = lowrank.lu_solve(A, B)
        assert np.linalg.norm(A @ X - B) / np.linalg.norm(B) < 1e-10


@pytest.mark.parametrize("precision,bound", [(0, 1e-13), (1, 2e-6), (2, 2e-6), (3, 2e-6), (4, 2e-6)])
@pytest.mark.parametrize("m,n,k,opA,opB", [
    (64, 64, 16, 0, 0), (1, 1, 1, 0, 0), (65, 33, 17, 1, 0), (200, 130, 451, 0, 1), (37, 300, 5, 1, 1),
    (10, 10, 0, 0, 0), (300, 260, 1000, 0, 0), (129, 257, 8, 1, 1), (100, 60, 2000, 1, 0),
])
def test_zgemm_precisions(precision, bound, m, n, k, opA, opB):
    """Grouped GEMM in FP64 and in split TF32 (FP32-level accuracy) against numpy.
    Launches of a few output tiles over long depths (200 x 130 x 451, 100 x 60
    x 2000) take the FP64 split-K path."""
    rng = np.random.default_rng(m * 7 + n * 3 + k)
    A = rng.standard_normal((k, m) if opA else (m, k)) + 1j * rng.standard_normal((k, m) if opA else (m, k))
    B = rng.standard_normal((n, k) if opB else (k, n)) + 1j * rng.standard_normal((n, k) if opB else (k, n))
    C0 = rng.standard_normal((m, n)) + 1j * rng.standard_normal((m, n))
    alpha, beta = 0.5 - 2j, 1.0 + 0.25j
    C = lowrank.zgemm(A, B, opA, opB, alpha, beta, C0, precision=precision)
    ref = alpha * ((A.conj().T if opA else A) @ (B.conj().T if opB else B)) + beta * C0
    scale = abs(alpha) * np.linalg.norm(A) * np.linalg.norm(B) + abs(beta) * np.linalg.norm(C0)
    assert np.linalg.norm(C - ref) <= bound * scale
    if precision >= 1 and k >= 16:  # split TF32 with FP32 accumulation, not an FP64 product
        assert np.linalg.norm(C - ref) >= 1e-12 * scale
    if precision >= 2:  # no tcgen05 pipeline wait ran out
        import ctypes as Cc
        from rcs_b200 import _lib
        n_to = Cc.c_long()
        _lib.check(_lib.lib().aifmm_tc5_timeouts(Cc.byref(n_to)))
        assert n_to.value == 0


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [2, 3, 4])
def test_tensor_core_wait_timeout_is_an_error(precision):
    """A tensor-core GEMM whose bounded wait runs out returns AIFMM_ETIMEOUT
    (not a silently unwritten C), and the context stays usable: the wait test
    holds every tile on a device flag that nothing sets, for at most 1 ms."""
    import ctypes as Cc
    from rcs_b200 import _lib
    from rcs_b200.kernel import Context
    ctx = Context(0)
    rng = np.random.default_rng(5)
    A = rng.standard_normal((200, 96)) + 1j * rng.standard_normal((200, 96))
    B = rng.standard_normal((96, 70)) + 1j * rng.standard_normal((96, 70))
    n0 = Cc.c_long()
    _lib.check(_lib.lib().aifmm_tc5_timeouts(Cc.byref(n0)))
    _lib.check(_lib.lib().aifmm_debug_gemm_hold(ctx.h, 1))
    try:
        with pytest.raises(RuntimeError) as e:
            lowrank.zgemm(A, B, precision=precision, ctx=ctx)
        assert "gave up" in str(e.value)
    finally:
        _lib.check(_lib.lib().aifmm_debug_gemm_hold(ctx.h, 0))
    n1 = Cc.c_long()
    _lib.check(_lib.lib().aifmm_tc5_timeouts(Cc.byref(n1)))
    # each tile (precision 2, 3: 2 row x 2 column tiles of 128 x 64) or each
    # persistent CTA (precision 4: 2 row x 1 column tiles of 128 x 128, one
    # CTA each) gave up once
    assert n1.value - n0.value == (2 if precision == 4 else 2 * 2)
    C = lowrank.zgemm(A, B, precision=precision, ctx=ctx)  # the same context afterwards
    assert np.linalg.norm(C - A @ B) <= 2e-6 * np.linalg.norm(A) * np.linalg.norm(B)
    ctx.close()


@pytest.mark.gpu
@pytest.mark.parametrize("form,raster", [(0, 1), (1, 0), (1, 1)])
@pytest.mark.parametrize("m,n,k,opA,opB", [(200, 130, 451, 0, 1), (300, 260, 1000, 0, 0), (129, 257, 8, 1, 1),
                                           (65, 33, 17, 1, 0)])
def test_persistent_gemm_forms(form, raster, m, n, k, opA, opB):
    """The persistent tensor-core GEMM in both operand forms and both tile
    orders: FP32-class accuracy, not an FP64 product, no wait ran out."""
    from rcs_b200.kernel import Context
    ctx = Context(0)
    ctx.set_gemm_tiling(form, raster)
    rng = np.random.default_rng(m + n + k)
    A = rng.standard_normal((k, m) if opA else (m, k)) + 1j * rng.standard_normal((k, m) if opA else (m, k))
    B = rng.standard_normal((n, k) if opB else (k, n)) + 1j * rng.standard_normal((n, k) if opB else (k, n))
    C0 = rng.standard_normal((m, n)) + 1j * rng.standard_normal((m, n))
    C = lowrank.zgemm(A, B, opA, opB, 0.5 - 2j, 1.0 + 0.25j, C0, precision=4, ctx=ctx)
    ref = (0.5 - 2j) * ((A.conj().T if opA else A) @ (B.conj().T if opB else B)) + (1.0 + 0.25j) * C0
    scale = abs(0.5 - 2j) * np.linalg.norm(A) * np.linalg.norm(B) + abs(1.0 + 0.25j) * np.linalg.norm(C0)
    assert 1e-12 * scale <= np.linalg.norm(C - ref) <= 2e-6 * scale
    ctx.close()
