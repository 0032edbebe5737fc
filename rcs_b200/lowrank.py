"""GPU low-rank and dense components with the reference's interfaces.

``ACA_only_nodes2`` mirrors LowRank<K>::ACA_only_nodes2 (src/ACA.cpp:639-859),
``RRQR`` mirrors RRQR::colPivHouseholderQRWithPartition (src/rrqr.cpp:3-182),
``lu_solve`` the dense partial-pivot LU solve of EFIEMatrix::getCoefficients
(src/EFIEMatrix.cpp:831-837).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .kernel import Context, default_context, kernel


def ACA_only_nodes2(K: kernel, rows, cols, tol: float):
    """Returns (row_bases, col_bases, Ac, Ar) with Ac = K(rows, cols[col_bases])
    and Ar = K(rows[row_bases], cols) (original, unreduced vectors)."""
    r = np.ascontiguousarray(rows, dtype=np.int32)
    c = np.ascontiguousarray(cols, dtype=np.int32)
    mn = min(len(r), len(c))
    rb = np.zeros(mn, dtype=np.int32)
    cb = np.zeros(mn, dtype=np.int32)
    Ac = np.zeros(2 * len(r) * mn, dtype=np.float64)
    Ar = np.zeros(2 * len(c) * mn, dtype=np.float64)
    rank = C.c_int()
    _lib.check(_lib.lib().aifmm_aca(K.h, r, len(r), c, len(c), float(tol), rb, cb, C.byref(rank), Ac, Ar))
    k = rank.value
    Acm = Ac[: 2 * len(r) * k].view(np.complex128).reshape(k, len(r)).T.copy()
    Arm = Ar[: 2 * len(c) * k].view(np.complex128).reshape(len(c), k).T.copy()
    return rb[:k].copy(), cb[:k].copy(), Acm, Arm


def RRQR(A: np.ndarray, tol_pow1: int, tol_pow2: int, partition: int, input_pivot: float, fill_rank: int,
         real_mode: bool = False, ctx: Context | None = None):
    """Returns (Q_trunc, maxPivot)."""
    ctx = ctx or default_context()
    A = np.asarray(A, dtype=np.complex128)
    m, n = A.shape
    flat = np.ascontiguousarray(A.T).ravel()
    Q = np.zeros(2 * m * min(m, n), dtype=np.float64)
    rank = C.c_int()
    mp = C.c_double()
    _lib.check(_lib.lib().aifmm_rrqr(ctx.h, flat.view(np.float64), m, n, int(partition), int(tol_pow1),
                                     int(tol_pow2), float(input_pivot), int(fill_rank), int(real_mode), Q,
                                     C.byref(rank), C.byref(mp)))
    k = rank.value
    return Q[: 2 * m * k].view(np.complex128).reshape(k, m).T.copy(), mp.value


def zgemm(A, B, opA=0, opB=0, alpha=1.0, beta=0.0, C=None, precision=0, ctx=None):
    """C = alpha op(A) op(B) + beta C on the GPU; op 1 = conjugate transpose;
    precision 1 = split-TF32 tensor cores (FP32 accuracy)."""
    ctx = ctx or default_context()
    A = np.asfortranarray(A, dtype=np.complex128)
    B = np.asfortranarray(B, dtype=np.complex128)
    m = A.shape[1] if opA else A.shape[0]
    k = A.shape[0] if opA else A.shape[1]
    n = B.shape[0] if opB else B.shape[1]
    Cm = np.zeros((m, n), dtype=np.complex128, order="F") if C is None else np.array(C, dtype=np.complex128, order="F")
    al = np.array([complex(alpha).real, complex(alpha).imag])
    be = np.array([complex(beta).real, complex(beta).imag])
    cflat = Cm.reshape(-1, order="F")  # a view: Cm is Fortran-ordered
    _lib.check(_lib.lib().aifmm_zgemm(ctx.h, int(precision), int(opA), int(opB), m, n, k, al,
                                      A.ravel(order="F").view(np.float64), max(A.shape[0], 1),
                                      B.ravel(order="F").view(np.float64), max(B.shape[0], 1), be,
                                      cflat.view(np.float64), max(m, 1)))
    return Cm


def lu_solve(A: np.ndarray, B: np.ndarray, ctx: Context | None = None) -> np.ndarray:
    ctx = ctx or default_context()
    A = np.asarray(A, dtype=np.complex128)
    B = np.asarray(B, dtype=np.complex128)
    one = B.ndim == 1
    B2 = B.reshape(A.shape[0], -1)
    n, nrhs = B2.shape
    X = np.zeros(n * nrhs, dtype=np.complex128)
    _lib.check(_lib.lib().aifmm_lu_solve(ctx.h, np.ascontiguousarray(A.T).ravel().view(np.float64), n,
                                         np.ascontiguousarray(B2.T).ravel().view(np.float64), nrhs,
                                         X.view(np.float64)))
    Xm = X.reshape(nrhs, n).T
    return Xm[:, 0].copy() if one else Xm.copy()
