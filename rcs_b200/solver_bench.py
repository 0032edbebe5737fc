"""Factor + solve timing of one sphere workload, with the phase breakdown.

    python -m rcs_b200.solver_bench [--sub 4] [--radius 0.15] [--freq 2e9] [--leaf 32]
                                    [--levels 3] [--tol-pow 5] [--fillin-tol 7]
                                    [--precision 0-4] [--drop-pow 0] [--op-tol 10] [--nrhs 8]
                                    [--gmres 1e-6] [--profile-ops] [--profile-host] [--profile-gemm]
                                    [--profiler-range] [--profile-solve]

Builds the EFIE operator of an icosphere (subdivision --sub), assembles the
AIFMM solver and, when --gmres is given, the FP64 H^2 forward operator; then
times one factorization and one solve (direct, or FGMRES to the target) and
prints one JSON line with the solver's phase timers.  A small, single-pass
workload for profiling the whole path (for example under a kernel profiler).
--profile-ops repeats the factorization and the solve with the library's
per-operation accounting on (every accounted operation then synchronises) and
prints its table.  --profiler-range brackets the timed factorization and
solve with cudaProfilerStart/Stop, so that a kernel profiler run with
capture from start off (ncu --profile-from-start off) records exactly their
launches.  --profile-solve times one direct solve issued launch by launch and
one replayed from the captured CUDA graph, then runs one more launch-by-launch
solve between cudaProfilerStart/Stop (for a launch list of the sweep).
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--sub", type=int, default=4)
    ap.add_argument("--radius", type=float, default=0.15)
    ap.add_argument("--freq", type=float, default=2.0e9)
    ap.add_argument("--leaf", type=int, default=32)
    ap.add_argument("--levels", type=int, default=3)
    ap.add_argument("--tol-pow", type=int, default=5)
    ap.add_argument("--fillin-tol", type=int, default=7)
    ap.add_argument("--precision", type=int, default=0)
    ap.add_argument("--drop-pow", type=int, default=0,
                    help="fill-in queue threshold 10^-k of the preconditioner (0: the reference's 10^-tol_pow)")
    ap.add_argument("--op-tol", type=int, default=10)
    ap.add_argument("--nrhs", type=int, default=8)
    ap.add_argument("--gmres", type=float, default=None)
    ap.add_argument("--profile-ops", action="store_true")
    ap.add_argument("--profile-gemm", action="store_true",
                    help="device time of the factorization's GEMM launches and RRQR chains by call site")
    ap.add_argument("--profile-host", action="store_true",
                    help="time the factorization with host-only accounting (no extra synchronisation)")
    ap.add_argument("--profiler-range", action="store_true",
                    help="cudaProfilerStart/Stop around the timed factorization and solve")
    ap.add_argument("--profile-solve", action="store_true",
                    help="time eager and graph-replayed direct solves; profiler range around one eager solve")
    a = ap.parse_args()
    from . import mesh as M
    from .kernel import EFIEMatrix
    from .solver import AIFMM, H2Operator
    K = EFIEMatrix(M.icosphere(a.sub, a.radius), a.freq)
    rng = np.random.default_rng(7)
    B = np.stack([K.planeWaveRhs(d / np.linalg.norm(d), np.cross(d, [0.3, 0.2, 0.9]).astype(complex))
                  for d in rng.standard_normal((a.nrhs, 3))], axis=1)
    t0 = time.perf_counter()
    S = AIFMM(K, leaf_size=a.leaf, tol_pow=a.tol_pow, fillin_tol=a.fillin_tol, n_levels=a.levels,
              precision=a.precision, drop_pow=a.drop_pow)
    t_asm = time.perf_counter() - t0
    if a.profile_ops:
        S.checkpoint()
    A = H2Operator(K, leaf_size=a.leaf, tol_pow=a.op_tol, n_levels=a.levels) if a.gmres else None
    if a.profile_host:
        from .solver import profile_ops
        profile_ops(2)
    if a.profile_gemm:
        from .solver import profile_gemm
        profile_gemm(True)
    if a.profiler_range:
        import torch
        torch.cuda.synchronize()
        torch.cuda.profiler.start()
    t0 = time.perf_counter()
    S.factorize()
    t_fac = time.perf_counter() - t0
    if a.profile_gemm:
        from .solver import profile_gemm, profile_gemm_table
        rows = profile_gemm_table()
        profile_gemm(False)
        tot = sum(r[2] for r in rows)
        print(f"# factorize: {t_fac:.3f} s; device time of the recorded launches {tot:.3f} s")
        print("| call site | launches | device s | TFLOP/s |\n|---|---|---|---|")
        for tag, n, sec, fl in sorted(rows, key=lambda r: -r[2]):
            print(f"| {tag} | {n} | {sec:.3f} | {fl / sec / 1e12 if sec > 0 and fl > 0 else 0:.1f} |")
    if a.profile_host:
        from .solver import profile_ops_read
        rows = [ln.split() for ln in profile_ops_read().strip().splitlines()]
        profile_ops(0)
        print(f"# factorize: {t_fac:.3f} s, host-time accounting (inclusive scopes, no extra synchronisation)")
        print("| operation | calls | host s |\n|---|---|---|")
        for r in sorted(rows, key=lambda r: -float(r[2])):
            print(f"| {r[0]} | {r[1]} | {float(r[2]):.3f} |")
    t0 = time.perf_counter()
    rec = None
    if A is not None:
        X, rec = S.solve_gmres(A, B, tol=a.gmres)
    else:
        X = S.solve(B)
    t_sol = time.perf_counter() - t0
    if a.profiler_range:
        torch.cuda.synchronize()
        torch.cuda.profiler.stop()
    if a.profile_solve:
        import torch
        times = {}
        for mode in (False, True):
            S.set_graph_solve(mode)
            S.solve(B)  # warm-up (the graph mode captures here)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            S.solve(B)
            times["graph" if mode else "eager"] = time.perf_counter() - t0
        S.set_graph_solve(False)
        torch.cuda.synchronize()
        torch.cuda.profiler.start()
        S.solve(B)
        torch.cuda.synchronize()
        torch.cuda.profiler.stop()
        S.set_graph_solve(True)
        print(f"# direct solve of {a.nrhs} right-hand sides: launch by launch {times['eager']:.4f} s, "
              f"graph replay {times['graph']:.4f} s")
    info = S.info()
    if a.precision == 5:
        for line in K.ctx.tune_report():
            print("# autotuner:", line)
    if a.profile_ops:
        from .solver import profile_ops, profile_ops_read
        S.rewind()
        for what, fn in (("factorize", S.factorize), ("solve", lambda: S.solve(B))):
            profile_ops(True)
            t0 = time.perf_counter()
            fn()
            dt = time.perf_counter() - t0
            rows = [ln.split() for ln in profile_ops_read().strip().splitlines()]
            profile_ops(False)
            print(f"# {what}: {dt:.3f} s with per-operation synchronisation")
            print("| operation | calls | s |\n|---|---|---|")
            for r in sorted(rows, key=lambda r: -float(r[2])):
                print(f"| {r[0]} | {r[1]} | {float(r[2]):.3f} |")
    print(json.dumps({"N": K.N, "precision": a.precision, "assemble_s": t_asm, "factor_s": t_fac, "solve_s": t_sol,
                      "gmres": rec, "phases_s": {k: v for k, v in info.items() if k.startswith("t_")},
                      "rrqr": info["n_rrqr"], "flops_factor": info["flops_factor"]}), flush=True)


if __name__ == "__main__":
    main()
