"""The AIFMM direct solver on the GPU, with the reference's interface.

``AIFMM`` mirrors vaishna77/RCS include/AIFMM.hpp:11-36: the constructor
builds the tree, the ACA skeletons, the M2L and leaf P2P blocks
(src/AIFMM.cpp:7-93); ``factorize`` runs the hierarchical elimination
(:96-100); ``solve`` = backSubstitute1/2/3 + getPhi (:103-147).  ``A`` exposes
the tree statistics that the reference's driver prints (getAvgLeafSize,
getAvgMultipoles, findMemory, findMemoryAfterFactorize, nLevels).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import _lib
from .kernel import kernel


class _TreeView:
    """Read-only stand-in for AIFMM::A (the FMM2DTree) as the driver uses it."""

    def __init__(self, solver: "AIFMM"):
        self._s = solver

    @property
    def nLevels(self) -> int:
        return self._s.info()["n_levels"]

    @property
    def K(self):
        return self._s.kernel

    def getAvgLeafSize(self) -> int:
        return self._s.info()["avg_leaf_size"]

    def getAvgMultipoles(self) -> int:
        return self._s.info()["avg_multipoles"]

    def findMemory(self) -> float:
        return self._s.info()["mem_gb"]

    def findMemoryAfterFactorize(self) -> float:
        return self._s.info()["mem_after_gb"]


class AIFMM:
    def __init__(self, K: kernel, leaf_size: int = 64, tol_pow: int = 8, fillin_tol: int = 10,
                 fillin_rank: int = 0, n_levels: int = 0, precision: int = 0, exact_rrqr: bool = False,
                 locations=None, domain=None, drop_pow: int = 0):
        """locations (N, 3) and domain (xmin, xmax, ymin, ymax, zmin, zmax) play
        the parts of inputsToSolverClass::locations and xmin..zmax; by default
        the tree is built over the kernel's own unknown locations.  drop_pow
        sets the fill-in queue threshold of a factorization used as a
        preconditioner (0: the reference's 10^-tol_pow; k > 0: 10^-k; negative:
        every well-separated fill-in is dropped)."""
        p = _lib.SolverParams(int(leaf_size), int(tol_pow), int(fillin_tol), int(fillin_rank), int(n_levels),
                              int(precision), int(bool(exact_rrqr)), int(drop_pow))
        h = C.c_void_p()
        if locations is None and domain is None:
            _lib.check(_lib.lib().aifmm_solver_create(K.h, C.byref(p), C.byref(h)))
        else:
            loc = np.ascontiguousarray(K.locations() if locations is None else locations, dtype=np.float64)
            if loc.shape != (K.N, 3):
                raise ValueError("locations must be (N, 3)")
            dom = None if domain is None else np.ascontiguousarray(domain, dtype=np.float64).reshape(6)
            _lib.check(_lib.lib().aifmm_solver_create_at(K.h, C.byref(p), loc.ravel(), K.N,
                                                          None if dom is None else dom.ctypes.data, C.byref(h)))
        self.h = h
        self.kernel = K
        self.N = K.N
        self.A = _TreeView(self)
        self._rhs = None

    def close(self):
        if getattr(self, "h", None):
            _lib.lib().aifmm_solver_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def factorize(self) -> None:
        _lib.check(_lib.lib().aifmm_solver_factorize(self.h))

    def solve(self, rhs) -> np.ndarray:
        """x for one (N,) or several (N, nrhs) right-hand sides."""
        b = np.asarray(rhs, dtype=np.complex128)
        one = b.ndim == 1
        B = b.reshape(self.N, -1)
        nrhs = B.shape[1]
        flat = np.ascontiguousarray(B.T).ravel()  # column-major N x nrhs
        X = np.zeros(self.N * nrhs, dtype=np.complex128)
        _lib.check(_lib.lib().aifmm_solver_solve(self.h, flat.view(np.float64), nrhs, X.view(np.float64)))
        Xm = X.reshape(nrhs, self.N).T
        return Xm[:, 0].copy() if one else Xm.copy()

    def set_graph_solve(self, on: bool) -> None:
        """Replay solves from a captured CUDA graph of the sweep (True, the default) or issue them launch by launch."""
        _lib.check(_lib.lib().aifmm_solver_set_graph_solve(self.h, 1 if on else 0))

    def solve_device(self, rhs_ptr: int, nrhs: int, x_ptr: int) -> None:
        _lib.check(_lib.lib().aifmm_solver_solve_device(self.h, C.c_void_p(rhs_ptr), int(nrhs), C.c_void_p(x_ptr)))

    # the reference's split of solve (src/AIFMM.cpp:120-147)
    def backSubstitute1(self, rhs) -> None:
        self._rhs = np.asarray(rhs, dtype=np.complex128)

    def backSubstitute2(self) -> None:
        pass  # the forward sweep runs inside backSubstitute3 (one device pass)

    def backSubstitute3(self) -> None:
        self._x = self.solve(self._rhs)

    def getPhi(self) -> np.ndarray:
        return self._x

    def solve_gmres(self, A: "H2Operator", rhs, tol: float = 1e-6, restart: int = 30,
                    maxit: int = 200) -> tuple[np.ndarray, dict]:
        """Flexible GMRES(restart) on the forward operator A, right-preconditioned
        by this factorization; returns x and the iteration record."""
        b = np.asarray(rhs, dtype=np.complex128)
        one = b.ndim == 1
        B = b.reshape(self.N, -1)
        nrhs = B.shape[1]
        flat = np.ascontiguousarray(B.T).ravel()
        X = np.zeros(self.N * nrhs, dtype=np.complex128)
        gi = _lib.GmresInfo()
        _lib.check(_lib.lib().aifmm_solver_solve_gmres(self.h, A.h, flat.view(np.float64), nrhs, X.view(np.float64),
                                                       float(tol), int(restart), int(maxit), C.byref(gi)))
        Xm = X.reshape(nrhs, self.N).T
        rec = {f: getattr(gi, f) for f, _ in gi._fields_}
        return (Xm[:, 0].copy() if one else Xm.copy()), rec

    def solve_gmres_device(self, A: "H2Operator", rhs_ptr: int, nrhs: int, x_ptr: int, tol: float = 1e-6,
                           restart: int = 30, maxit: int = 200) -> dict:
        gi = _lib.GmresInfo()
        _lib.check(_lib.lib().aifmm_solver_solve_gmres_device(self.h, A.h, C.c_void_p(rhs_ptr), int(nrhs),
                                                              C.c_void_p(x_ptr), float(tol), int(restart),
                                                              int(maxit), C.byref(gi)))
        return {f: getattr(gi, f) for f, _ in gi._fields_}

    def tree_order(self) -> np.ndarray:
        """order[p] = the unknown at position p of the tree-ordered solution
        (FMM2DTree::getx before reorder)."""
        out = np.zeros(self.N, dtype=np.int32)
        _lib.check(_lib.lib().aifmm_solver_tree_order(self.h, out))
        return out

    def info(self) -> dict:
        i = _lib.SolverInfo()
        _lib.check(_lib.lib().aifmm_solver_get_info(self.h, C.byref(i)))
        return {f: getattr(i, f) for f, _ in i._fields_}

    def dump(self) -> np.ndarray:
        """(n, 7) array: level, box, kind, key, rows, cols, Frobenius norm per block."""
        cnt = C.c_long()
        _lib.check(_lib.lib().aifmm_solver_dump(self.h, None, 0, C.byref(cnt)))
        out = np.zeros(7 * cnt.value, dtype=np.float64)
        _lib.check(_lib.lib().aifmm_solver_dump(self.h, out.ctypes.data, cnt.value, C.byref(cnt)))
        return out.reshape(-1, 7)

    def checkpoint(self) -> None:
        """Keep a device copy of the assembled operator (before factorize)."""
        _lib.check(_lib.lib().aifmm_solver_checkpoint(self.h))

    def save(self, path: str) -> None:
        """Write the factorization to a checkpoint file (aifmm_solver_save)."""
        _lib.check(_lib.lib().aifmm_solver_save(self.h, os.fsencode(path)))

    @classmethod
    def load(cls, K: kernel, path: str) -> "AIFMM":
        """A solver on kernel K with the factorization read from a checkpoint
        file (aifmm_solver_load): it solves without assembly or factorization."""
        self = cls.__new__(cls)
        h = C.c_void_p()
        _lib.check(_lib.lib().aifmm_solver_load(K.h, os.fsencode(path), C.byref(h)))
        self.h = h
        self.kernel = K
        self.N = K.N
        self.A = _TreeView(self)
        self._rhs = None
        return self

    def rewind(self) -> None:
        """Restore the checkpointed operator so that factorize can run again."""
        _lib.check(_lib.lib().aifmm_solver_rewind(self.h))


class H2Operator:
    """FP64 forward operator y = A x of the kernel in H^2 form: the assembly of
    AIFMM (octree, ACA skeletons, L2P/P2M, M2L, leaf P2P) at ACA tolerance
    10^-tol_pow, kept unfactorized.  The residual operator of
    AIFMM.solve_gmres; the reference has no counterpart."""

    def __init__(self, K: kernel, leaf_size: int = 64, tol_pow: int = 10, n_levels: int = 0):
        p = _lib.SolverParams(int(leaf_size), int(tol_pow), int(tol_pow), 0, int(n_levels), 0, 0)
        h = C.c_void_p()
        _lib.check(_lib.lib().aifmm_operator_create(K.h, C.byref(p), C.byref(h)))
        self.h = h
        self.N = K.N

    def close(self):
        if getattr(self, "h", None):
            _lib.lib().aifmm_operator_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __matmul__(self, x) -> np.ndarray:
        b = np.asarray(x, dtype=np.complex128)
        one = b.ndim == 1
        B = b.reshape(self.N, -1)
        nrhs = B.shape[1]
        flat = np.ascontiguousarray(B.T).ravel()
        Y = np.zeros(self.N * nrhs, dtype=np.complex128)
        _lib.check(_lib.lib().aifmm_operator_apply(self.h, flat.view(np.float64), nrhs, Y.view(np.float64)))
        Ym = Y.reshape(nrhs, self.N).T
        return Ym[:, 0].copy() if one else Ym.copy()

    def apply_device(self, x_ptr: int, nrhs: int, y_ptr: int) -> None:
        _lib.check(_lib.lib().aifmm_operator_apply_device(self.h, C.c_void_p(x_ptr), int(nrhs), C.c_void_p(y_ptr)))

    def info(self) -> dict:
        b, f = C.c_double(), C.c_double()
        _lib.check(_lib.lib().aifmm_operator_info(self.h, C.byref(b), C.byref(f)))
        return {"bytes": b.value, "flops_per_column": f.value}


def launch_count() -> int:
    n = C.c_long()
    _lib.check(_lib.lib().aifmm_launch_count(C.byref(n)))
    return n.value


def profile_ops(on) -> None:
    """Start (clear) or stop the per-operation accounting of the solver:
    False/0 off; True/1 every accounted operation synchronises (host enqueue +
    device time); 2 host time only, plus the time blocked on the device
    (sync_wait, ring_wait) and in the memory pool (pool_alloc, pool_free)."""
    mode = 1 if on is True else (0 if on is False else int(on))
    _lib.check(_lib.lib().aifmm_profile_ops(mode))


def profile_ops_read() -> str:
    buf = C.create_string_buffer(1 << 16)
    _lib.check(_lib.lib().aifmm_profile_ops_read(buf, len(buf)))
    return buf.value.decode()


def profile_gemm(on: bool) -> None:
    _lib.check(_lib.lib().aifmm_profile_gemm(int(bool(on))))


def profile_gemm_table() -> list[tuple[str, int, float, float]]:
    """Device time by call site while the GEMM profiler is on: (tag, launches,
    seconds, flops) for the grouped GEMMs ("gemm:<precision>:<scope path>") and
    the RRQR launch chains ("rrqr:<scope path>")."""
    buf = C.create_string_buffer(1 << 20)
    _lib.check(_lib.lib().aifmm_profile_gemm_table(buf, len(buf)))
    out = []
    for ln in buf.value.decode().strip().splitlines():
        tag, n, sec, fl = ln.rsplit(" ", 3)
        out.append((tag, int(n), float(sec), float(fl)))
    return out


def profile_gemm_read() -> tuple[float, float, int]:
    ms, fl, n = C.c_double(), C.c_double(), C.c_long()
    _lib.check(_lib.lib().aifmm_profile_gemm_read(C.byref(ms), C.byref(fl), C.byref(n)))
    return ms.value, fl.value, n.value
