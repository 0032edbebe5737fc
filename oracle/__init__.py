"""CPU oracle for the AIFMM hot path -- TEST INFRASTRUCTURE ONLY.

A C++ restatement of vaishna77/RCS (EFIE/electrostatics entries, ACA, RRQR,
the H^2 tree, its elimination and solve sweeps), loaded through ctypes.  Only
``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this package, and only as the checker; the product
library never links it.

Parity status: pinned against outputs of the reference itself.  The
reference's unmodified sources build here against the project-written Eigen
subset (oracle/ref.mk, oracle/ref_driver.cpp); tests/golden/make_ref_golden.py
records their outputs as tests/golden/ref_*.npz and tests/test_oracle_ref_pin.py
checks this oracle against them: bit-identical where the factorization makes
no fill-in recompression, identical ranks of every box and the solution within
the RRQR tolerance (two levels) or the ACA tolerance (three levels) where it
does.  The oracle is also pinned against known answers: dense LU on the same
operator, the analytic sphere capacitance, the Mie series of a PEC sphere,
RRQR/ACA residuals and the H^2 approximation error.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None

_i = C.c_int
_d = C.c_double
_p = C.c_void_p
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_lp = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (g++, no GPU needed)."""
    if force or not os.path.exists(_LIB_PATH):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def build_ref(root: str | None = None) -> str | None:
    """Compile the reference itself into oracle/_ref/aifmm_ref (oracle/ref.mk)
    when its source tree is present: AIFMM_REFERENCE_ROOT, else the build
    container's mount at /root/reference.  Returns the binary, or None when the
    tree is absent (the GPU box has only what was built beforehand)."""
    root = root or os.environ.get("AIFMM_REFERENCE_ROOT") or "/root/reference"
    if not os.path.isdir(os.path.join(root, "src")):
        return None
    subprocess.run(["make", "-s", "-f", os.path.join(_HERE, "ref.mk"), f"REF={root}", "-j8"], check=True,
                   cwd=os.path.dirname(_HERE))
    return os.path.join(_HERE, "_ref", "aifmm_ref")


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(_LIB_PATH)
        sig = {
            "or_last_error": (C.c_char_p, []),
            "or_set_threads": (None, [_i]),
            "or_get_threads": (_i, []),
            "or_efie_create": (_p, [_dp, _i, _ip, _i, _d, _i]),
            "or_es_create": (_p, [_dp, _i, _ip, _i, _ip]),
            "or_kernel_destroy": (None, [_p]),
            "or_kernel_n": (_i, [_p]),
            "or_kernel_matrix": (_i, [_p, _ip, _i, _ip, _i, _dp]),
            "or_kernel_locations": (_i, [_p, _dp]),
            "or_efie_rwg": (_i, [_p, _ip, _dp]),
            "or_efie_rhs_reference": (_i, [_p, _dp, _dp]),
            "or_efie_rhs_plane": (_i, [_p, _dp, _dp, _dp]),
            "or_dense_solve": (_i, [_p, _dp, _i, _dp]),
            "or_aca": (_i, [_p, _ip, _i, _ip, _i, _d, _ip, _ip, _dp, _dp]),
            "or_rrqr": (_i, [_dp, _i, _i, _i, _i, _i, _d, _i, _i, _dp, _dp, _ip, _dp, _dp]),
            "or_lu_solve": (_i, [_dp, _i, _dp, _i, _dp]),
            "or_aifmm_create": (_p, [_p, _dp, _i, _i, _i, _i, _i, _dp, _i]),
            "or_aifmm_destroy": (None, [_p]),
            "or_aifmm_factorize": (_i, [_p]),
            "or_aifmm_solve": (_i, [_p, _dp, _dp]),
            "or_aifmm_info": (_i, [_p, _lp, _dp, _dp]),
            "or_aifmm_leaf_counts": (_i, [_p, _ip]),
            "or_efie_set_plane_projection": (None, [_p, _i]),
            "or_aifmm_dump": (C.c_long, [_p, _p, C.c_long]),
            "or_tree_shape_create": (_p, [_p, _dp, _i, _i, _dp]),
            "or_tree_shape_sizes": (None, [_p, _ip]),
            "or_tree_shape_get": (None, [_p, _ip, _ip, _ip, _ip]),
            "or_tree_shape_destroy": (None, [_p]),
            "or_schur_sample": (_i, [_p, _ip, _i, _ip, _ip, _i, _ip, _i, _i, _dp, _dp]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _check(rc):
    if rc is None or (isinstance(rc, int) and rc < 0):
        raise RuntimeError("oracle: " + lib().or_last_error().decode())
    return rc


def _c2d(z: np.ndarray) -> np.ndarray:
    """complex128 array -> interleaved float64 (column-major for matrices)."""
    z = np.asarray(z, dtype=np.complex128)
    return np.ascontiguousarray(np.asfortranarray(z).ravel(order="F").view(np.float64))


def set_threads(n: int) -> None:
    lib().or_set_threads(int(n))


class Kernel:
    def __init__(self, handle, kind: str):
        if not handle:
            raise RuntimeError("oracle: " + lib().or_last_error().decode())
        self.h = handle
        self.kind = kind
        self.N = lib().or_kernel_n(handle)

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.or_kernel_destroy(self.h)
            self.h = None

    def matrix(self, rows, cols) -> np.ndarray:
        r = np.ascontiguousarray(rows, dtype=np.int32)
        c = np.ascontiguousarray(cols, dtype=np.int32)
        out = np.zeros(2 * len(r) * len(c), dtype=np.float64)
        _check(lib().or_kernel_matrix(self.h, r, len(r), c, len(c), out))
        return out.view(np.complex128).reshape((len(c), len(r))).T.copy()

    def dense(self) -> np.ndarray:
        idx = np.arange(self.N, dtype=np.int32)
        return self.matrix(idx, idx)

    def locations(self) -> np.ndarray:
        out = np.zeros(3 * self.N, dtype=np.float64)
        lib().or_kernel_locations(self.h, out)
        return out.reshape(self.N, 3)

    def dense_solve(self, rhs: np.ndarray) -> np.ndarray:
        b = np.asarray(rhs, dtype=np.complex128)
        if b.ndim == 1:
            b = b[:, None]
        out = np.zeros(2 * b.size, dtype=np.float64)
        _check(lib().or_dense_solve(self.h, _c2d(b), b.shape[1], out))
        return out.view(np.complex128).reshape((b.shape[1], self.N)).T.squeeze()


class EFIE(Kernel):
    def __init__(self, mesh, freq: float = 1.0e7, exact_lookup: bool = False):
        nodes = np.ascontiguousarray(mesh.nodes, dtype=np.float64).ravel()
        tris = np.ascontiguousarray(mesh.tris, dtype=np.int32).ravel()
        h = lib().or_efie_create(nodes, mesh.n_nodes, tris, mesh.n_tris, float(freq), int(exact_lookup))
        super().__init__(h, "efie")
        self.freq = freq

    def set_plane_projection(self, on: bool) -> None:
        lib().or_efie_set_plane_projection(self.h, int(bool(on)))

    def rwg(self):
        t = np.zeros(6 * self.N, dtype=np.int32)
        ln = np.zeros(self.N, dtype=np.float64)
        lib().or_efie_rwg(self.h, t, ln)
        return t.reshape(self.N, 6), ln

    def rhs_reference(self, einc=(1.0, 0.0, 0.0)) -> np.ndarray:
        out = np.zeros(2 * self.N, dtype=np.float64)
        lib().or_efie_rhs_reference(self.h, np.asarray(einc, dtype=np.float64), out)
        return out.view(np.complex128).copy()

    def rhs_plane(self, khat, e0) -> np.ndarray:
        out = np.zeros(2 * self.N, dtype=np.float64)
        e = np.asarray(e0, dtype=np.complex128).view(np.float64)
        lib().or_efie_rhs_plane(self.h, np.asarray(khat, dtype=np.float64), np.ascontiguousarray(e), out)
        return out.view(np.complex128).copy()


class Electrostatics(Kernel):
    def __init__(self, mesh):
        nodes = np.ascontiguousarray(mesh.nodes, dtype=np.float64).ravel()
        tris = np.ascontiguousarray(mesh.tris, dtype=np.int32).ravel()
        cond = mesh.cond if mesh.cond is not None else np.ones(mesh.n_tris, dtype=np.int32)
        h = lib().or_es_create(nodes, mesh.n_nodes, tris, mesh.n_tris, np.ascontiguousarray(cond, dtype=np.int32))
        super().__init__(h, "es")


def aca(kernel: Kernel, rows, cols, tol: float):
    r = np.ascontiguousarray(rows, dtype=np.int32)
    c = np.ascontiguousarray(cols, dtype=np.int32)
    m = min(len(r), len(c))
    rb = np.zeros(max(m, 1), dtype=np.int32)
    cb = np.zeros(max(m, 1), dtype=np.int32)
    Ac = np.zeros(2 * len(r) * max(m, 1), dtype=np.float64)
    Ar = np.zeros(2 * len(c) * max(m, 1), dtype=np.float64)
    k = _check(lib().or_aca(kernel.h, r, len(r), c, len(c), float(tol), rb, cb, Ac, Ar))
    Acm = Ac[: 2 * len(r) * k].view(np.complex128).reshape((k, len(r))).T
    Arm = Ar[: 2 * len(c) * k].view(np.complex128).reshape((len(c), k)).T
    return rb[:k].copy(), cb[:k].copy(), Acm.copy(), Arm.copy()


def rrqr(A: np.ndarray, tolpow1: int, tolpow2: int, partition: int, input_pivot: float, fill_rank: int,
         real_mode: bool = False):
    A = np.asarray(A, dtype=np.complex128)
    m, n = A.shape
    Q = np.zeros(2 * m * m, dtype=np.float64)
    R = np.zeros(2 * m * n, dtype=np.float64)
    perm = np.zeros(n, dtype=np.int32)
    mp = np.zeros(1)
    err = np.zeros(1)
    k = _check(lib().or_rrqr(_c2d(A), m, n, tolpow1, tolpow2, partition, float(input_pivot), fill_rank,
                             int(real_mode), Q, R, perm, mp, err))
    Qm = Q[: 2 * m * k].view(np.complex128).reshape((k, m)).T.copy()
    Rm = R[: 2 * k * n].view(np.complex128).reshape((n, k)).T.copy()
    return Qm, Rm, perm, float(mp[0]), float(err[0])


class AIFMM:
    """The reference's AIFMM<K> facade over the oracle tree."""

    def __init__(self, kernel: Kernel, leaf_size: int, tol_pow: int, fillin_tol: int, fillin_rank: int = 0,
                 n_levels: int = 0, locations: np.ndarray | None = None):
        loc = kernel.locations() if locations is None else np.asarray(locations, dtype=np.float64)
        bbox = np.array([loc[:, 0].min(), loc[:, 0].max(), loc[:, 1].min(), loc[:, 1].max(),
                         loc[:, 2].min(), loc[:, 2].max()], dtype=np.float64)
        self.kernel = kernel
        self.N = kernel.N
        self.h = lib().or_aifmm_create(kernel.h, bbox, int(leaf_size), int(tol_pow), int(n_levels),
                                       int(fillin_rank), int(fillin_tol), np.ascontiguousarray(loc).ravel(),
                                       int(kernel.kind == "es"))
        if not self.h:
            raise RuntimeError("oracle: " + lib().or_last_error().decode())

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.or_aifmm_destroy(self.h)
            self.h = None

    def factorize(self):
        _check(lib().or_aifmm_factorize(self.h))

    def solve(self, rhs: np.ndarray) -> np.ndarray:
        out = np.zeros(2 * self.N, dtype=np.float64)
        _check(lib().or_aifmm_solve(self.h, _c2d(np.asarray(rhs, dtype=np.complex128)), out))
        return out.view(np.complex128).copy()

    def dump(self) -> np.ndarray:
        """(n, 7) array: level, box, kind, key, rows, cols, Frobenius norm per block."""
        n = lib().or_aifmm_dump(self.h, None, 0)
        out = np.zeros(7 * n, dtype=np.float64)
        lib().or_aifmm_dump(self.h, out.ctypes.data, n)
        return out.reshape(-1, 7)

    def info(self) -> dict:
        i = np.zeros(8, dtype=np.int64)
        t = np.zeros(3)
        m = np.zeros(2)
        lib().or_aifmm_info(self.h, i, t, m)
        return dict(nLevels=int(i[0]), startLevel=int(i[1]), avgLeafSize=int(i[2]), avgMultipoles=int(i[3]),
                    maxRank=int(i[4]), nRRQR=int(i[5]), nCompressP2P=int(i[6]), nCompressP2L=int(i[7]),
                    t_assemble=float(t[0]), t_factor=float(t[1]), t_solve=float(t[2]),
                    mem_GB=float(m[0]), mem_after_GB=float(m[1]))


def tree_shape(kernel: Kernel, leaf_size: int, n_levels: int = 0):
    """The reference's tree over the kernel's locations without skeletons:
    (n_levels, leaf point lists, leaf neighbour lists), leaves in box order."""
    loc = kernel.locations()
    bbox = np.array([loc[:, 0].min(), loc[:, 0].max(), loc[:, 1].min(), loc[:, 1].max(),
                     loc[:, 2].min(), loc[:, 2].max()], dtype=np.float64)
    h = lib().or_tree_shape_create(kernel.h, bbox, int(leaf_size), int(n_levels), np.ascontiguousarray(loc).ravel())
    if not h:
        raise RuntimeError("oracle: " + lib().or_last_error().decode())
    try:
        sz = np.zeros(3, dtype=np.int32)
        lib().or_tree_shape_sizes(h, sz)
        nl, nleaf, nnb = (int(v) for v in sz)
        po = np.zeros(nleaf + 1, dtype=np.int32)
        pts = np.zeros(max(kernel.N, 1), dtype=np.int32)
        no = np.zeros(nleaf + 1, dtype=np.int32)
        nbi = np.zeros(max(nnb, 1), dtype=np.int32)
        lib().or_tree_shape_get(h, po, pts, no, nbi)
    finally:
        lib().or_tree_shape_destroy(h)
    leaves = [pts[po[b]:po[b + 1]].copy() for b in range(nleaf)]
    nbs = [nbi[no[b]:no[b + 1]].copy() for b in range(nleaf)]
    return nl, leaves, nbs


def schur_sample(kernel: Kernel, box_pts, nb_pts: list, pairs, threads: int):
    """Times the reference's leaf-level near-field Schur updates of one box
    (LU of P2P[k][k]; P2P[nn][pp] -= P2P[nn][k] lu.solve(P2P[k][pp]) per pair)
    on `threads` threads.  Returns (seconds_lu, seconds_pairs, macs_lu,
    macs_pairs)."""
    bp = np.ascontiguousarray(box_pts, dtype=np.int32)
    off = np.zeros(len(nb_pts) + 1, dtype=np.int32)
    off[1:] = np.cumsum([len(v) for v in nb_pts])
    flat = np.ascontiguousarray(np.concatenate(nb_pts) if nb_pts else np.zeros(1), dtype=np.int32)
    pr = np.ascontiguousarray(np.asarray(pairs, dtype=np.int32).ravel())
    sec = np.zeros(2)
    macs = np.zeros(2)
    _check(lib().or_schur_sample(kernel.h, bp, len(bp), off, flat, len(nb_pts), pr, len(pr) // 2, int(threads), sec,
                                 macs))
    return float(sec[0]), float(sec[1]), float(macs[0]), float(macs[1])
