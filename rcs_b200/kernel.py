"""Matrix-entry kernels on the GPU, with the reference's interface.

``EFIEMatrix`` and ``ElectrostaticsMatrix`` mirror vaishna77/RCS
include/EFIEMatrix.hpp and include/ElectrostaticsMatrix.hpp on top of
``kernel`` (include/kernel.hpp:13-47): ``N``, ``getMatrixEntry``, ``getRow``,
``getCol``, ``getMatrix`` (index lists or a contiguous range), ``getRhs``.
All entries are computed by the CUDA kernels of libaifmm_b200.so.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .mesh import Mesh


class Context:
    """One GPU, one CUDA stream and a device memory pool (aifmm_ctx)."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        _lib.check(_lib.lib().aifmm_ctx_create(int(device), C.byref(h)))
        self.h = h
        self.device = device

    def synchronize(self):
        _lib.check(_lib.lib().aifmm_ctx_synchronize(self.h))

    def stream(self) -> int:
        s = C.c_void_p()
        _lib.check(_lib.lib().aifmm_ctx_stream(self.h, C.byref(s)))
        return s.value or 0

    def set_gemm_tiling(self, form: int = 0, raster: int = 0) -> None:
        """Operand form (0 packed real, 1 split planes) and tile order (0
        row-major, 1 column-major) of GEMM precision 4 on this context."""
        _lib.check(_lib.lib().aifmm_ctx_set_gemm_tiling(self.h, int(form), int(raster)))

    def memory(self) -> dict:
        """Bytes held by the context's buffers (live) and by its memory pool (reserved)."""
        live, res = C.c_size_t(), C.c_size_t()
        _lib.check(_lib.lib().aifmm_ctx_memory(self.h, C.byref(live), C.byref(res)))
        return {"live": live.value, "reserved": res.value}

    def trim(self) -> None:
        """Return the context's unused device memory (free arena chunks, pooled blocks) to the device."""
        _lib.check(_lib.lib().aifmm_ctx_trim(self.h))

    def tune_report(self) -> list[str]:
        """The GEMM autotuner's trials on this context, one line per launch
        class (GEMM precision 5)."""
        n = C.c_int()
        _lib.check(_lib.lib().aifmm_ctx_tune_report(self.h, None, 0, C.byref(n)))
        buf = C.create_string_buffer(n.value + 1)
        _lib.check(_lib.lib().aifmm_ctx_tune_report(self.h, buf, n.value + 1, C.byref(n)))
        return [ln for ln in buf.value.decode().splitlines() if ln]

    def close(self):
        if getattr(self, "h", None):
            _lib.lib().aifmm_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_default_ctx: Context | None = None


def default_context() -> Context:
    global _default_ctx
    if _default_ctx is None:
        _default_ctx = Context(0)
    return _default_ctx


class kernel:
    """Base of the GPU matrix-entry kernels (include/kernel.hpp)."""

    def __init__(self, handle: C.c_void_p, ctx: Context):
        self.h = handle
        self.ctx = ctx
        n = C.c_int()
        _lib.check(_lib.lib().aifmm_kernel_size(self.h, C.byref(n)))
        self.N = n.value

    def close(self):
        if getattr(self, "h", None):
            _lib.lib().aifmm_kernel_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # kernel::getMatrix(row_indices, col_indices), src/kernel.cpp:49-61
    def getMatrix(self, rows, cols=None, rows_end=None, cols_end=None, precision: int = 0) -> np.ndarray:
        if cols is not None and rows_end is not None:  # getMatrix(r0, c0, r1, c1), src/kernel.cpp:63-73
            rows, cols = np.arange(rows, rows_end), np.arange(cols, cols_end)
        r = np.ascontiguousarray(rows, dtype=np.int32)
        c = np.ascontiguousarray(cols, dtype=np.int32)
        dt = np.complex128 if precision == 0 else np.complex64
        out = np.zeros((len(c), len(r)), dtype=dt)  # C-order (nc, nr) == column-major (nr, nc)
        if len(r) and len(c):
            _lib.check(_lib.lib().aifmm_kernel_matrix(self.h, r, len(r), c, len(c), int(precision),
                                                      out.ctypes.data, len(r)))
        return out.T

    def getRow(self, i: int, cols) -> np.ndarray:  # src/kernel.cpp:11-19
        return self.getMatrix([i], cols)[0]

    def getCol(self, j: int, rows) -> np.ndarray:  # src/kernel.cpp:21-29
        return self.getMatrix(rows, [j])[:, 0]

    def getMatrixEntry(self, i: int, j: int) -> complex:
        return complex(self.getMatrix([i], [j])[0, 0])

    def dense(self, precision: int = 0) -> np.ndarray:
        idx = np.arange(self.N, dtype=np.int32)
        return self.getMatrix(idx, idx, precision=precision)

    def locations(self) -> np.ndarray:
        out = np.zeros(3 * self.N, dtype=np.float64)
        _lib.check(_lib.lib().aifmm_kernel_locations(self.h, out))
        return out.reshape(self.N, 3)


class EFIEMatrix(kernel):
    """EFIE (RWG) kernel: EFIEMatrix(inputsToKernelClass), src/EFIEMatrix.cpp:5-20."""

    def __init__(self, mesh: Mesh, freq: float = 1.0e7, ctx: Context | None = None):
        ctx = ctx or default_context()
        nodes = np.ascontiguousarray(mesh.nodes, dtype=np.float64).ravel()
        tris = np.ascontiguousarray(mesh.tris, dtype=np.int32).ravel()
        h = C.c_void_p()
        _lib.check(_lib.lib().aifmm_kernel_create_efie(ctx.h, nodes, mesh.n_nodes, tris, mesh.n_tris, float(freq),
                                                        C.byref(h)))
        super().__init__(h, ctx)
        self.freq = freq
        self.mesh = mesh

    def setPlaneProjection(self, on: bool) -> None:
        """False (default): the reference's projection quirk; True: project the
        test point onto the source triangle's plane (Mie-accurate)."""
        _lib.check(_lib.lib().aifmm_kernel_set_plane_projection(self.h, int(bool(on))))

    def getRhs(self, Einc=(1.0, 0.0, 0.0)) -> np.ndarray:
        """EFIEMatrix::getRhs(Node& Einc, VectorXcd& rhs), src/EFIEMatrix.cpp:785-829."""
        out = np.zeros(2 * self.N, dtype=np.float64)
        _lib.check(_lib.lib().aifmm_kernel_rhs_reference(self.h, np.asarray(Einc, dtype=np.float64), out))
        return out.view(np.complex128).copy()

    def planeWaveRhs(self, khat, e0) -> np.ndarray:
        """Physical plane wave E0 exp(-i k khat.r) (khat: propagation direction)."""
        out = np.zeros(2 * self.N, dtype=np.float64)
        e = np.ascontiguousarray(np.asarray(e0, dtype=np.complex128).view(np.float64))
        _lib.check(_lib.lib().aifmm_kernel_rhs_plane(self.h, np.asarray(khat, dtype=np.float64), e, out))
        return out.view(np.complex128).copy()


    def getJAtCentroids(self, coefficients) -> np.ndarray:
        """Surface current at the triangle centroids, (n_tris, 3) complex:
        EFIEMatrix::getJAtCentroids, src/EFIEMatrix.cpp:1100-1130 (on the GPU)."""
        c = np.ascontiguousarray(np.asarray(coefficients, dtype=np.complex128).reshape(self.N)).view(np.float64)
        out = np.zeros(6 * self.mesh.n_tris, dtype=np.float64)
        _lib.check(_lib.lib().aifmm_kernel_currents(self.h, c, out))
        return out.view(np.complex128).reshape(3, self.mesh.n_tris).T.copy()

    def getRCS_OnePointQuadrature(self, theta, phi, J) -> np.ndarray:
        """Bistatic RCS of centroid currents J at the angles (theta, phi)
        (arrays of equal length, or scalars): EFIEMatrix::getRCS_OnePointQuadrature,
        src/EFIEMatrix.cpp:916-930, all angles in one GPU launch."""
        th = np.atleast_1d(np.asarray(theta, dtype=np.float64))
        ph = np.broadcast_to(np.asarray(phi, dtype=np.float64), th.shape)
        Jc = np.asarray(J, dtype=np.complex128)
        if Jc.shape != (self.mesh.n_tris, 3):
            raise ValueError("J must be (n_tris, 3)")
        Jf = np.ascontiguousarray(Jc.T).view(np.float64).ravel()
        out = np.zeros(th.size, dtype=np.float64)
        _lib.check(_lib.lib().aifmm_kernel_rcs(self.h, Jf, th.size, np.ascontiguousarray(th),
                                                np.ascontiguousarray(ph), out))
        return out


class ElectrostaticsMatrix(kernel):
    """Piecewise-constant collocation kernel, src/ElectrostaticsMatrix.cpp:48-52."""

    def __init__(self, mesh: Mesh, ctx: Context | None = None):
        ctx = ctx or default_context()
        nodes = np.ascontiguousarray(mesh.nodes, dtype=np.float64).ravel()
        tris = np.ascontiguousarray(mesh.tris, dtype=np.int32).ravel()
        cond = np.ascontiguousarray(mesh.cond if mesh.cond is not None else np.ones(mesh.n_tris), dtype=np.int32)
        h = C.c_void_p()
        _lib.check(_lib.lib().aifmm_kernel_create_es(ctx.h, nodes, mesh.n_nodes, tris, cond.ctypes.data,
                                                      mesh.n_tris, C.byref(h)))
        super().__init__(h, ctx)
        self.mesh = mesh

    def getRhs(self, conductor: int = 1) -> np.ndarray:
        """ElectrostaticsMatrix::getRhs(conductorIndex, rhs), :374-381."""
        out = np.zeros(2 * self.N, dtype=np.float64)
        _lib.check(_lib.lib().aifmm_kernel_rhs_conductor(self.h, int(conductor), out))
        return out.view(np.complex128).real.copy()
