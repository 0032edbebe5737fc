"""aifmm_rrqr_noalloc: the RRQR entry point for callers that cannot allocate
device memory (another framework owns the allocator, a stream is being
captured, or the memory budget is reserved up front).  It takes only device
pointers and keeps its working storage in a fixed device array of the
library, so it is checked here against the allocating aifmm_rrqr on two calls
in a row (the second reuses the array the first left behind).

This file is collected last on purpose: it must pass both on its own in a
fresh process and after every other test.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _case(seed, m, r0, nf, frank):
    rng = np.random.default_rng(seed)
    U = (rng.standard_normal((m, r0)) + 1j * rng.standard_normal((m, r0))) * np.logspace(0, -12, r0)[None, :]
    F = (rng.standard_normal((m, frank)) + 1j * rng.standard_normal((m, frank))) @ \
        (rng.standard_normal((frank, nf)) + 1j * rng.standard_normal((frank, nf)))
    return np.hstack([U, F])


def _noalloc(A, tp1, tp2, part, pivot, fill):
    import torch
    from rcs_b200 import _lib
    m, n = A.shape
    # inputs and outputs are the caller's device buffers (allocated here by the test)
    Ad = torch.from_numpy(np.ascontiguousarray(A.T)).cuda()  # column-major m x n
    Qd = torch.zeros((min(m, n), m), dtype=torch.complex128, device="cuda")
    rk = torch.zeros(1, dtype=torch.int32, device="cuda")
    mp = torch.zeros(1, dtype=torch.float64, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    _lib.check(_lib.lib().aifmm_rrqr_noalloc(C.c_void_p(Ad.data_ptr()), m, n, part, tp1, tp2, float(pivot), fill,
                                             0, C.c_void_p(Qd.data_ptr()), C.c_void_p(rk.data_ptr()),
                                             C.c_void_p(mp.data_ptr()), C.c_void_p(s)))
    torch.cuda.synchronize()
    r = int(rk.item())
    return Qd.cpu().numpy()[:r].T, float(mp.item()), Ad.cpu().numpy().T


def test_noalloc_rrqr_matches_allocating_entry_point_twice():
    from rcs_b200 import lowrank
    cases = [(11, 60, 10, 30, 8, 8, 10, 5, 10.0), (12, 45, 7, 50, 12, 10, 9, 10, 0.5)]
    for seed, m, r0, nf, frank, tp1, tp2, fill, pivot in cases:  # two calls in a row
        A = _case(seed, m, r0, nf, frank)
        Q, mp, A_after = _noalloc(A, tp1, tp2, r0, pivot, fill)
        Qr, mpr = lowrank.RRQR(A, tp1, tp2, r0, pivot, fill)
        assert np.array_equal(A_after, A)  # the input is not modified
        assert Q.shape == Qr.shape
        assert abs(mp - mpr) <= 1e-12 * max(mpr, 1.0)
        assert np.linalg.norm(Q - Qr) <= 1e-10 * max(np.linalg.norm(Qr), 1.0)


def test_noalloc_rrqr_rejects_oversized_problem():
    import torch
    from rcs_b200 import _lib
    from rcs_b200._lib import AifmmError
    m = n = 1500  # needs more than the 32 MiB scratch
    Ad = torch.zeros((n, m), dtype=torch.complex128, device="cuda")
    Qd = torch.zeros((n, m), dtype=torch.complex128, device="cuda")
    rk = torch.zeros(1, dtype=torch.int32, device="cuda")
    mp = torch.zeros(1, dtype=torch.float64, device="cuda")
    with pytest.raises(AifmmError):
        _lib.check(_lib.lib().aifmm_rrqr_noalloc(C.c_void_p(Ad.data_ptr()), m, n, 10, 8, 8, 1.0, 5, 0,
                                                 C.c_void_p(Qd.data_ptr()), C.c_void_p(rk.data_ptr()),
                                                 C.c_void_p(mp.data_ptr()), None))


def test_noalloc_rrqr_captures_in_a_cuda_graph():
    """The property the entry point exists for: after a first call, a call
    allocates nothing and can be captured in a CUDA graph; replays give the
    eager call's results bit for bit and leave the input untouched."""
    import torch
    from rcs_b200 import _lib
    seed, m, r0, nf, frank, tp1, tp2, fill, pivot = (11, 60, 10, 30, 8, 8, 10, 5, 10.0)
    A = _case(seed, m, r0, nf, frank)
    Q_ref, mp_ref, _ = _noalloc(A, tp1, tp2, r0, pivot, fill)  # the first call looks up the scratch array
    n = A.shape[1]
    Ad = torch.from_numpy(np.ascontiguousarray(A.T)).cuda()
    Qd = torch.zeros((min(m, n), m), dtype=torch.complex128, device="cuda")
    rk = torch.zeros(1, dtype=torch.int32, device="cuda")
    mp = torch.zeros(1, dtype=torch.float64, device="cuda")

    def call(stream):
        _lib.check(_lib.lib().aifmm_rrqr_noalloc(C.c_void_p(Ad.data_ptr()), m, n, r0, tp1, tp2, float(pivot), fill,
                                                 0, C.c_void_p(Qd.data_ptr()), C.c_void_p(rk.data_ptr()),
                                                 C.c_void_p(mp.data_ptr()), C.c_void_p(stream)))

    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    call(torch.cuda.current_stream().cuda_stream)  # an eager call after the first: no device allocation
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    Qd.zero_()
    rk.zero_()
    mp.zero_()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        call(torch.cuda.current_stream().cuda_stream)
    for _ in range(2):
        g.replay()
        torch.cuda.synchronize()
        r = int(rk.item())
        assert np.array_equal(Qd.cpu().numpy()[:r].T, Q_ref) and float(mp.item()) == mp_ref
    assert np.array_equal(Ad.cpu().numpy().T, A)
