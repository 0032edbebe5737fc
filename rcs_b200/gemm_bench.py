"""Throughput of the library's complex GEMM kernels on one GPU.

    python -m rcs_b200.gemm_bench [--m 2048 --n 2048 --k 2048] [--precision 0 1 2]
                                  [--reps 20] [--batch 1]

Times C = A B (complex128 storage) through aifmm_zgemm_device with CUDA events
on the library's stream, after warm-up, and prints one JSON line per
precision: 0 = FP64 FMA (zgemm_grouped_kernel), 1 = split TF32 on the tensor
cores by mma.sync, 2 = split TF32 by tcgen05 with tensor-memory accumulators
and the split inside the tile loop, 3 = the same with the operands split once
into pre-tiled planes that the tile loop streams with bulk copies, 4 = the
persistent warp-specialised kernel (--form, --raster), 5 = the autotuner's
choice.
Flops are complex-counted (8 m n k per product).  --batch B issues B
independent products per launch (the grouped form the solver uses).  The
operands total more than the 126 MB L2 for the default size with --batch 8.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json

import numpy as np


def run(m: int, n: int, k: int, precision: int, reps: int = 20, batch: int = 1, device: int = 0, form: int = 0,
        raster: int = 0) -> dict:
    """form, raster: the persistent kernel's operand form and tile order
    (precision 4; the library's defaults are 1 and 0)."""
    import torch
    from . import _lib
    from .kernel import Context
    torch.cuda.set_device(device)
    ctx = Context(device)
    ctx.set_gemm_tiling(form, raster)
    stream = torch.cuda.ExternalStream(ctx.stream(), device=device)
    g = torch.Generator(device=f"cuda:{device}").manual_seed(1)
    A = [torch.randn(k, m, dtype=torch.complex128, device=f"cuda:{device}", generator=g) for _ in range(batch)]
    B = [torch.randn(n, k, dtype=torch.complex128, device=f"cuda:{device}", generator=g) for _ in range(batch)]
    Cs = [torch.zeros(n, m, dtype=torch.complex128, device=f"cuda:{device}") for _ in range(batch)]
    al = np.array([1.0, 0.0])
    be = np.array([0.0, 0.0])
    torch.cuda.synchronize()

    def once():
        for q in range(batch):  # column-major m x k / k x n / m x n views of the row-major tensors
            _lib.check(_lib.lib().aifmm_zgemm_device(ctx.h, precision, 0, 0, m, n, k, al, C.c_void_p(A[q].data_ptr()),
                                                     m, C.c_void_p(B[q].data_ptr()), k, be,
                                                     C.c_void_p(Cs[q].data_ptr()), m))

    for _ in range(3):
        once()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        once()
    e1.record(stream)
    torch.cuda.synchronize()
    sec = e0.elapsed_time(e1) / 1e3 / reps
    # accuracy of the last product against a complex128 reference on a few columns
    ref = (A[0].T @ B[0].T[:, :8])
    got = Cs[0].T[:, :8]
    err = float(torch.linalg.norm(got - ref) / torch.linalg.norm(ref))
    return {"m": m, "n": n, "k": k, "batch": batch, "precision": precision, "form": form, "raster": raster,
            "seconds": sec,
            "tflops": 8.0 * m * n * k * batch / sec / 1e12, "rel_err": err}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--m", type=int, default=2048)
    ap.add_argument("--n", type=int, default=2048)
    ap.add_argument("--k", type=int, default=2048)
    ap.add_argument("--precision", type=int, nargs="+", default=[0, 1, 2, 3])
    ap.add_argument("--reps", type=int, default=20)
    ap.add_argument("--batch", type=int, default=1)
    ap.add_argument("--form", type=int, default=1, help="precision 4: 0 packed real, 1 split planes (default)")
    ap.add_argument("--raster", type=int, default=0, help="precision 4: 0 row-major, 1 column-major tile order")
    a = ap.parse_args()
    for p in a.precision:
        print(json.dumps(run(a.m, a.n, a.k, p, a.reps, a.batch, form=a.form, raster=a.raster)), flush=True)


if __name__ == "__main__":
    main()
