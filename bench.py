#!/usr/bin/env python
"""Benchmark of the AIFMM factor+solve on B200.

One step = factorize + solve of the assembled EFIE operator (the checkpointed
assembly is restored on the device at the start of each step, inside the
timed region).  The metric is the reference's: seconds of factor+solve at the
stated relative residual.  Prints one JSON line (rank 0).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--config c3] [--impl reference]

Under torchrun each rank runs an independent replica of the workload on its
own GPU (one geometry does not shard: replicas only); the step time is the
maximum over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "factor+solve s at rel. residual 1e-6: mixed/batched/learned vs plain FP64 GPU"

# Workloads (the benchmark configurations); synthetic icosphere meshes, seeded plane waves.
# tol_pow / fillin_tol: the factorization's ACA and RRQR tolerances; op_tol:
# ACA tolerance of the FP64 H^2 forward operator that GMRES iterates on; gmres:
# target relative residual (None = direct solve only, the reference's path).
CONFIGS = {
    "c1": dict(N=1920, sub=3, radius=0.15, freq=1.0e9, leaf=64, tol_pow=8, fillin_tol=10, nrhs=1, levels=0, op_tol=None,
               gmres=None, precision=0,
               desc="EFIE PEC sphere R=0.15 m f=1 GHz, 1,280 tri, N=1,920, leaf 64, ACA 1e-8, RRQR 1e-10, "
                    "direct solve"),
    "c3": dict(N=122880, sub=6, radius=0.15, freq=4.0e9, leaf=128, tol_pow=5, fillin_tol=7, nrhs=8, levels=0, op_tol=9,
               gmres=1e-6, precision=4, drop_pow=1,
               desc="EFIE PEC sphere R=0.15 m f=4 GHz (ka=12.6), 81,920 tri, N=122,880, leaf 128, ACA 1e-5, "
                    "RRQR 1e-7, 8 seeded plane waves, mixed factorization (split-TF32 persistent tcgen05 GEMMs; "
                    "fill-ins under 1e-1 of their M2L block dropped) as the preconditioner of FP64 FGMRES(30) to "
                    "1e-6 on an ACA-1e-9 H2 operator"),
    "c2": dict(N=81920, kind="es", sub=6, radius=1.0, leaf=128, tol_pow=5, fillin_tol=7, nrhs=33, levels=0,
               op_tol=10, gmres=1e-8, precision=4, drop_pow=1,
               desc="Electrostatics unit sphere, 81,920 flat triangles (piecewise-constant charge, collocation at "
                    "centroids), leaf 128, ACA 1e-5, RRQR 1e-7, 32 seeded N(0,1) potentials + the 1 V conductor "
                    "RHS, mixed factorization (split-TF32 tcgen05 GEMMs, FP32-class) as the preconditioner of FP64 "
                    "FGMRES(30) to 1e-8 on an ACA-1e-10 H2 operator; capacitance vs 4 pi eps0 R"),
    "c3s": dict(N=30720, sub=5, radius=0.15, freq=2.0e9, leaf=32, tol_pow=5, fillin_tol=7, nrhs=8, levels=0, op_tol=10,
                gmres=1e-6, precision=4, drop_pow=1,
                desc="EFIE PEC sphere R=0.15 m f=2 GHz, 20,480 tri, N=30,720, leaf 32, ACA 1e-5, RRQR 1e-7, "
                     "8 plane waves, FGMRES(30) to 1e-6 (c3 shape at 1/4 size)"),
}
# Batched bodies: 64 seeded ellipsoids (semi-axes U[0.05, 0.3] m), icosphere
# subdivisions 3 and 4 alternating (1,920 and 7,680 unknowns), 2 GHz, 4 plane
# waves each; every body on its own context, factorized and refined
# concurrently (aifmm_batch_factorize / aifmm_batch_solve_gmres).
BATCH = dict(bodies=64, seed=64, subdivisions=(3, 4), freq=2.0e9, leaf=32, tol_pow=5, fillin_tol=7, nrhs=4,
             op_tol=12, gmres=1e-6, precision=4, drop_pow=2, threads=16,
             desc="Batched EFIE: 64 PEC ellipsoids, semi-axes U[0.05,0.3] m (seed 64), icosphere 3/4 alternating "
                  "(1,920 / 7,680 unknowns), f=2 GHz, 4 plane waves each, leaf 32, ACA 1e-5, RRQR 1e-7; mixed "
                  "factorization (split-TF32 tcgen05) refined by FP64 FGMRES(30) to 1e-6 on an ACA-1e-12 H2 operator "
                  "(at 1e-10 the operator error, amplified by ||x||/||b|| ~ 140 near resonance, left two bodies at "
                  "5e-6), bodies on concurrent streams")
# CPU baseline (reference arm and cpu_baseline): pair updates per timed sample.
CPU_PAIRS_PER_SAMPLE = 16


def plane_waves(n: int, seed: int = 4):
    """Seeded incidence directions uniform on the sphere (theta = acos(1-2u),
    phi = 2 pi u), alternating theta/phi polarisation."""
    rng = np.random.Generator(np.random.MT19937(seed))
    out = []
    for q in range(n):
        th = math.acos(1 - 2 * rng.random())
        ph = 2 * math.pi * rng.random()
        k = np.array([math.sin(th) * math.cos(ph), math.sin(th) * math.sin(ph), math.cos(th)])
        e_th = np.array([math.cos(th) * math.cos(ph), math.cos(th) * math.sin(ph), -math.sin(th)])
        e_ph = np.array([-math.sin(ph), math.cos(ph), 0.0])
        out.append((k, (e_th if q % 2 == 0 else e_ph).astype(np.complex128)))
    return out


def es_rhs(K, n_random: int, seed: int = 20261203) -> np.ndarray:
    """Electrostatics right-hand sides: n_random seeded N(0,1) potential
    vectors (one per column) and the 1 V conductor right-hand side last
    (ElectrostaticsMatrix::getRhs)."""
    rng = np.random.Generator(np.random.MT19937(seed))
    R = rng.standard_normal((K.N, n_random))
    return np.concatenate([R, K.getRhs(1)[:, None]], axis=1).astype(np.complex128)


def capacitance_error(mesh, sigma: np.ndarray, radius: float) -> float:
    """C / (4 pi eps0 R) - 1 for the 1 V charge density (getCapacitance,
    src/ElectrostaticsMatrix.cpp:366-402: total charge over the potential)."""
    v = mesh.nodes[mesh.tris - 1]
    area = 0.5 * np.linalg.norm(np.cross(v[:, 1] - v[:, 0], v[:, 2] - v[:, 0]), axis=1)
    return float(np.real(sigma) @ area) / (4 * np.pi * 8.854187817e-12 * radius) - 1.0


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, device: int):
        self.device = device
        self.rows = []
        self.proc = None

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if len(r) > 3 + i and r[3 + i] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def max_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def build_workload(cfg, device: int):
    """Mesh, kernel, right-hand sides, the assembled (checkpointed) solver and,
    when the config refines, the FP64 forward operator.  Not timed as a step:
    the reference times assembly separately from factor+solve."""
    from rcs_b200 import mesh as M
    from rcs_b200.kernel import Context, EFIEMatrix, ElectrostaticsMatrix
    from rcs_b200.solver import AIFMM, H2Operator
    ctx = Context(device)
    m = M.icosphere(cfg["sub"], cfg["radius"])
    if cfg.get("kind", "efie") == "es":
        K = ElectrostaticsMatrix(m, ctx=ctx)
        B = es_rhs(K, cfg["nrhs"] - 1)
    else:
        K = EFIEMatrix(m, cfg["freq"], ctx=ctx)
        waves = plane_waves(cfg["nrhs"]) if cfg["nrhs"] > 1 else [(np.array([0.0, 0, -1]), np.array([1, 0, 0j]))]
        B = np.stack([K.planeWaveRhs(k, e) for k, e in waves], axis=1)
    t0 = time.perf_counter()
    S = AIFMM(K, leaf_size=cfg["leaf"], tol_pow=cfg["tol_pow"], fillin_tol=cfg["fillin_tol"], n_levels=cfg["levels"],
              precision=cfg.get("precision", 0), drop_pow=cfg.get("drop_pow", 0))
    t_asm = time.perf_counter() - t0
    S.checkpoint()
    A, t_op = None, 0.0
    if cfg.get("op_tol") is not None:
        t0 = time.perf_counter()
        A = H2Operator(K, leaf_size=cfg["leaf"], tol_pow=cfg["op_tol"], n_levels=cfg["levels"])
        t_op = time.perf_counter() - t0
    return ctx, m, K, S, A, B, t_asm, t_op


def sampled_residual(K, X: np.ndarray, B: np.ndarray, nrows: int = 2048, seed: int = 1) -> float:
    """||A x - b|| / ||b|| over a seeded sample of rows (full rows of A on the GPU)."""
    rng = np.random.default_rng(seed)
    rows = np.sort(rng.choice(K.N, size=min(nrows, K.N), replace=False))
    acc = np.zeros((len(rows), X.shape[1]), dtype=np.complex128)
    for c0 in range(0, K.N, 16384):
        cols = np.arange(c0, min(K.N, c0 + 16384))
        acc += K.getMatrix(rows, cols) @ X[cols]
    r = acc - B[rows]
    return float(np.linalg.norm(r) / np.linalg.norm(B[rows]))


def zgemm_peak_tflops() -> float:
    """cuBLAS complex128 GEMM throughput on this GPU (the FP64 denominator)."""
    import torch
    n = 4096
    a = torch.randn(n, n, dtype=torch.complex128, device="cuda")
    b = torch.randn(n, n, dtype=torch.complex128, device="cuda")
    for _ in range(2):
        a @ b
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    best = 1e30
    for _ in range(5):
        e0.record()
        a @ b
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1) / 1e3)
    return 8.0 * n ** 3 / best / 1e12


class CPUBaseline:
    """The reference's CPU algorithm (the oracle, a C++ restatement; the
    reference itself needs Eigen 3, absent here) on the benchmark's own tree.

    The full factorization of the 122,880-unknown sphere takes hours on the
    host, so one sample times a bounded piece of it: for one leaf box k of the
    workload's tree, the LU of its near-field block and up to
    CPU_PAIRS_PER_SAMPLE of the near-field Schur updates that the
    reference's eliminate_x performs for it (P2P[nn][pp] -= P2P[nn][k]
    lu.solve(P2P[k][pp]) for neighbours nn, pp not yet eliminated, the solve
    recomputed per pair as the reference does), at the workload's block
    sizes.  The extrapolation multiplies the measured seconds per complex
    multiply-add by the multiply-adds of every such update of the leaf level,
    counted from the tree's box sizes and neighbour lists in elimination
    order, plus three LUs per leaf box (the factorization's and the two of
    the reference's solve).  It leaves out the rank-sized updates, eliminate_z,
    the recompressions, the non-leaf level and the assembly, so it is a LOWER
    BOUND on the reference's factor+solve time."""

    def __init__(self, cfg):
        import oracle
        from rcs_b200 import mesh as M
        self.oracle = oracle
        self.cfg = cfg
        m = M.icosphere(cfg["sub"], cfg["radius"])
        self.K = oracle.EFIE(m, cfg["freq"]) if cfg.get("kind", "efie") == "efie" else oracle.Electrostatics(m)
        self.n_levels, self.leaves, self.nbs = oracle.tree_shape(self.K, cfg["leaf"], cfg["levels"])
        sizes = np.array([len(v) for v in self.leaves], dtype=np.float64)
        self.lu_macs = 0.0
        self.pair_macs = 0.0
        self.n_pairs = 0
        self.cands = []
        for k, mk in enumerate(sizes):
            if mk == 0:
                continue
            self.lu_macs += 3 * mk ** 3 / 3.0
            live = [nn for nn in self.nbs[k] if nn != k and nn > k and sizes[nn] > 0]
            for nn in live:
                for pp in live:
                    self.pair_macs += mk * mk * sizes[pp] + sizes[nn] * mk * sizes[pp]
                    self.n_pairs += 1
            if live:
                self.cands.append(k)
        self.order = np.random.default_rng(20261204).permutation(len(self.cands))
        self.samples = []

    def sample(self, i: int, threads: int):
        """Sample i: (seconds, lu seconds, pair seconds, lu macs, pair macs)."""
        k = self.cands[self.order[i % len(self.order)]]
        sizes = [len(v) for v in self.leaves]
        live = [nn for nn in self.nbs[k] if nn != k and nn > k and sizes[nn] > 0]
        pairs = [(a, b) for a in range(len(live)) for b in range(len(live))]
        rng = np.random.default_rng(i)
        if len(pairs) > CPU_PAIRS_PER_SAMPLE:
            pairs = [pairs[q] for q in sorted(rng.choice(len(pairs), CPU_PAIRS_PER_SAMPLE, replace=False))]
        s_lu, s_pairs, m_lu, m_pairs = self.oracle.schur_sample(self.K, self.leaves[k],
                                                               [self.leaves[nn] for nn in live], pairs, threads)
        r = dict(box=int(k), m=sizes[k], pairs=len(pairs), s_lu=s_lu, s_pairs=s_pairs, m_lu=m_lu, m_pairs=m_pairs)
        return s_lu + s_pairs, r

    @staticmethod
    def extrapolate(recs, lu_macs, pair_macs) -> float:
        s_lu = sum(r["s_lu"] for r in recs)
        s_p = sum(r["s_pairs"] for r in recs)
        m_lu = sum(r["m_lu"] for r in recs)
        m_p = sum(r["m_pairs"] for r in recs)
        return lu_macs * s_lu / m_lu + pair_macs * s_p / m_p

    def describe(self, recs, threads: int) -> str:
        return (f"oracle (C++ restatement of the reference) on the workload's own tree ({self.n_levels} levels, "
                f"{len(self.cands)} leaf boxes with near-field updates, {self.n_pairs} updates in elimination "
                f"order): {len(recs)} timed samples on {threads} thread(s), each one leaf box's near-field LU "
                f"and up to {CPU_PAIRS_PER_SAMPLE} of its pair updates at the workload's block sizes "
                f"({sum(r['s_lu'] + r['s_pairs'] for r in recs):.1f} s timed); extrapolated by complex "
                f"multiply-adds to every leaf near-field update and three LUs per leaf box "
                f"({(self.lu_macs + self.pair_macs) / 1e12:.2f} T multiply-adds).  A lower bound: rank-sized "
                f"updates, eliminate_z, recompressions, the non-leaf level and assembly are not counted")


def peaks():
    """MEASURED_PEAKS.json (driver-written, measured on this pool's B200s) or
    the recorded fallback figures of this pool."""
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return {"hbm_gbs": float(d["hbm_gbs"]), "bf16_tflops": float(d["bf16_tflops"]),
                "bf16_tflops_sustained": float(d.get("bf16_tflops_sustained", d["bf16_tflops"])),
                "source": "measured (MEASURED_PEAKS.json)"}
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0,
                "source": "fallback (earlier measurement on this pool; MEASURED_PEAKS.json absent)"}


def config_block(cfg, world):
    """The `config` object of both arms (identical, so the driver can pair them)."""
    return {"workload": cfg["desc"], "N": cfg.get("N"), "nrhs": cfg["nrhs"],
            "parallelism": "replicas" if world > 1 else "single GPU",
            "l2": "inputs larger than L2 (leaf blocks and fill-ins stream from HBM)"}


def run_reference(args, rank, world):
    """Reference arm: the reference's CPU algorithm (the oracle) on the host
    cores, all threads, on bounded samples of the workload's own tree,
    extrapolated to the workload (a lower bound; see CPUBaseline).  Loads no
    GPU library.  Rank 0 only."""
    if rank != 0:
        return
    if args.config not in CONFIGS:
        print(json.dumps({"impl": "reference", "metric": METRIC, "config": {"workload": args.config},
                          "unavailable": "the reference arm is measured on the single-geometry configurations "
                                         "(c1, c2, c3, c3s); the batched one has no CPU run of its own"}), flush=True)
        return
    cfg = CONFIGS[args.config]
    threads = os.cpu_count() or 1
    t_setup = time.perf_counter()
    cb = CPUBaseline(cfg)
    t_setup = time.perf_counter() - t_setup
    for i in range(args.warmup):
        cb.sample(i, threads)
    recs = []
    t0 = time.perf_counter()
    for i in range(args.steps):
        recs.append(cb.sample(args.warmup + i, threads)[1])
    t_timed = time.perf_counter() - t0
    v = cb.extrapolate(recs, cb.lu_macs, cb.pair_macs)
    # the reference factorizes on one thread (test/sphere.cpp:206-207): one more sample at 1 thread
    r1 = cb.sample(args.warmup + args.steps, 1)[1]
    v1 = cb.extrapolate([r1], cb.lu_macs, cb.pair_macs)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": v * 1e3, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "c128", "data": "synthetic", "config": config_block(cfg, world),
            "extrapolated": "lower bound",
            "reference_path": "the reference's factorization (the oracle restates it; Eigen 3 is absent) on the host "
                              "CPU; no refinement",
            "cpu_baseline": {"value": v, "unit": "s", "cores": threads, "kind": "port",
                             "sample": cb.describe(recs, threads)},
            "single_thread": {"value": v1, "unit": "s", "cores": 1, "sample": cb.describe([r1], 1)},
            "samples": recs, "timed_region_s": t_timed, "setup_s": t_setup,
            "e2e": {"value": v, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_batch(args, rank, world, local):
    """The batched-bodies workload: all bodies' factorizations and FGMRES
    solves per step, concurrently; beside it the same bodies one after another
    on the plain FP64 path."""
    import torch
    from rcs_b200 import batch
    from rcs_b200.kernel import Context, EFIEMatrix
    from rcs_b200.solver import AIFMM, H2Operator, launch_count
    torch.cuda.set_device(local)
    cfg = BATCH
    bodies = []
    t0 = time.perf_counter()
    for mesh, axes in batch.ellipsoid_family(cfg["bodies"], cfg["seed"], cfg["subdivisions"]):
        ctx = Context(local)
        K = EFIEMatrix(mesh, cfg["freq"], ctx=ctx)
        B = np.stack([K.planeWaveRhs(k, e) for k, e in plane_waves(cfg["nrhs"])], axis=1)
        S = AIFMM(K, leaf_size=cfg["leaf"], tol_pow=cfg["tol_pow"], fillin_tol=cfg["fillin_tol"],
                  precision=cfg["precision"], drop_pow=cfg["drop_pow"])
        S.checkpoint()
        A = H2Operator(K, leaf_size=cfg["leaf"], tol_pow=cfg["op_tol"])
        ctx.trim()  # the assembly's temporaries go back to the device for the next bodies
        bodies.append(dict(ctx=ctx, K=K, S=S, A=A, B=B, axes=axes))
    t_setup = time.perf_counter() - t0
    Ss, As, Bs = [b["S"] for b in bodies], [b["A"] for b in bodies], [b["B"] for b in bodies]
    stream = torch.cuda.Stream(device=local)
    out = {}

    def step():
        for S in Ss:
            S.rewind()
        tf = batch.batch_factorize(Ss, threads=cfg["threads"])
        xs, recs, ts = batch.batch_solve_gmres(Ss, As, Bs, tol=cfg["gmres"], maxit=300, threads=cfg["threads"])
        out.update(xs=xs, recs=recs, tf=tf, ts=ts)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    barrier(world)
    l0 = launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        e0.record(stream)
        t_f = t_s = 0.0
        for _ in range(args.steps):
            step()  # returns after every body's stream has drained
            t_f += out["tf"]
            t_s += out["ts"]
        e1.record(stream)
        torch.cuda.synchronize()
    launches = launch_count() - l0
    t_step = max_over_ranks(e0.elapsed_time(e1) / 1e3 / args.steps, world)
    mem = [b["ctx"].memory() for b in bodies]
    res = [sampled_residual(b["K"], x, b["B"], nrows=256) for b, x in zip(bodies, out["xs"])]
    for b in bodies:  # the batch's factorizations go before the plain path's, one body at a time
        b["S"].close()
        b["ctx"].trim()
    # the plain FP64 path, one body after another (one timed pass)
    plain = None
    if not args.no_plain:
        t0 = time.perf_counter()
        its = []
        for b in bodies:
            S0 = AIFMM(b["K"], leaf_size=cfg["leaf"], tol_pow=cfg["tol_pow"], fillin_tol=cfg["fillin_tol"],
                       precision=0)
            torch.cuda.synchronize()
            f0 = time.perf_counter()
            S0.factorize()
            _, rec = S0.solve_gmres(b["A"], b["B"], tol=cfg["gmres"], maxit=300)
            torch.cuda.synchronize()
            its.append((time.perf_counter() - f0, rec["iterations"]))
            S0.close()
        plain = {"value": float(sum(t for t, _ in its)), "unit": "s", "gmres_iterations_mean": float(np.mean(
            [i for _, i in its])), "mode": "bodies one after another, plain complex128 factorization + FGMRES"}
    if rank == 0:
        Ns = [b["K"].N for b in bodies]
        line = {
            "metric": METRIC, "value": t_step, "unit": "s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_step * 1e3, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "c128+tf32x3", "data": "synthetic",
            "config": {"workload": cfg["desc"], "bodies": len(bodies), "N_total": int(sum(Ns)),
                       "N_min": int(min(Ns)), "N_max": int(max(Ns)), "nrhs": cfg["nrhs"],
                       "parallelism": "replicas" if world > 1 else "single GPU"},
            "factor_s": t_f / args.steps, "solve_s": t_s / args.steps,
            "residual_max": float(max(res)), "residual_per_body": [float(r) for r in res],
            "gmres_iterations": [r["iterations"] for r in out["recs"]],
            "plain_fp64": plain, "setup_s": t_setup, "gpu_launches": int(launches), "clocks": clk.summary(),
            "device_gb_after_step": {"live": sum(m["live"] for m in mem) / 1e9,
                                     "reserved": sum(m["reserved"] for m in mem) / 1e9,
                                     "operators": sum(b["A"].info()["bytes"] for b in bodies) / 1e9},
            "e2e": {"value": t_step, "unit": "s", "h2d_bytes_per_step": int(16 * sum(Ns) * cfg["nrhs"]),
                    "d2h_bytes_per_step": int(16 * sum(Ns) * cfg["nrhs"]),
                    "note": "the batch entry points take host right-hand sides and return host solutions"},
        }
        print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--config", default=os.environ.get("AIFMM_BENCH_CONFIG", "c3"))
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain FP64 comparison step")
    args = ap.parse_args()
    rank, world, local = dist_env()
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("gloo", timeout=timedelta(seconds=900))
    if args.impl == "reference":
        run_reference(args, rank, world)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    if args.config == "c4":
        run_batch(args, rank, world, local)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    import torch
    torch.cuda.set_device(local)
    from rcs_b200.solver import launch_count, profile_gemm, profile_gemm_table
    cfg = CONFIGS[args.config]
    ctx, m, K, S, A, B, t_asm, t_op = build_workload(cfg, local)
    N, nrhs = K.N, B.shape[1]
    assert N == cfg["N"], "the mesh does not have the configuration's unknown count"
    stream = torch.cuda.ExternalStream(ctx.stream(), device=local)
    Bd = torch.from_numpy(np.ascontiguousarray(B.T)).to(f"cuda:{local}")  # nrhs x N == column-major N x nrhs
    Xd = torch.empty_like(Bd)
    recs = []

    def step():
        S.rewind()
        S.factorize()
        if A is None:
            S.solve_device(Bd.data_ptr(), nrhs, Xd.data_ptr())
        else:
            recs.append(S.solve_gmres_device(A, Bd.data_ptr(), nrhs, Xd.data_ptr(), tol=cfg["gmres"], restart=30,
                                             maxit=300))

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    barrier(world)
    recs.clear()
    l0 = launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(args.steps):
            step()
        e1.record(stream)
        torch.cuda.synchronize()
    launches = launch_count() - l0
    barrier(world)
    t_step = max_over_ranks(e0.elapsed_time(e1) / 1e3 / args.steps, world)
    X = Xd.cpu().numpy().T
    res = sampled_residual(K, X, B)
    info = S.info()
    gm = None
    if recs:
        gm = {"iterations_per_step": [r["iterations"] for r in recs], "relres_operator": max(r["relres"] for r in recs),
              "precond_s_per_step": float(np.mean([r["t_precond"] for r in recs])),
              "matvec_s_per_step": float(np.mean([r["t_matvec"] for r in recs]))}

    # e2e: the public host API, pinned host buffers, H2D/D2H inside the step
    # (a few steps: the same work as `value`, through the host-buffer call)
    Bh = torch.from_numpy(np.ascontiguousarray(B.T)).pin_memory()
    Xh = torch.empty_like(Bh).pin_memory()
    from rcs_b200 import _lib
    import ctypes as C
    hb = np.ctypeslib.as_array(C.cast(Bh.data_ptr(), C.POINTER(C.c_double)), shape=(2 * N * nrhs,))
    hx = np.ctypeslib.as_array(C.cast(Xh.data_ptr(), C.POINTER(C.c_double)), shape=(2 * N * nrhs,))
    e2e_steps = min(args.steps, 3)
    barrier(world)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        S.rewind()
        _lib.check(_lib.lib().aifmm_solver_factorize(S.h))
        if A is None:
            _lib.check(_lib.lib().aifmm_solver_solve(S.h, hb, nrhs, hx))
        else:
            gi = _lib.GmresInfo()
            _lib.check(_lib.lib().aifmm_solver_solve_gmres(S.h, A.h, hb, nrhs, hx, float(cfg["gmres"]), 30, 300,
                                                           C.byref(gi)))
    t_e2e = max_over_ranks((time.perf_counter() - t0) / e2e_steps, world)
    res_e2e = sampled_residual(K, Xh.numpy().T, B, nrows=512)

    # device time of every grouped-GEMM launch and RRQR chain of one more
    # step, by call site (CUDA events on the library stream around each launch)
    profile_gemm(True)
    step()
    torch.cuda.synchronize()
    table = profile_gemm_table()
    profile_gemm(False)
    pk = peaks()
    zpeak = zgemm_peak_tflops()
    phases = {}
    for tag, n, sec, fl in table:
        if not tag.startswith("gemm:"):
            continue
        prec = int(tag.split(":")[1])
        key = "tcgen05 split-TF32 GEMM" if prec >= 2 else "FP64 GEMM"
        ph = phases.setdefault(key, {"launches": 0, "device_s": 0.0, "flops": 0.0})
        ph["launches"] += n
        ph["device_s"] += sec
        ph["flops"] += fl
    for key, ph in phases.items():
        ph["tflops"] = ph["flops"] / ph["device_s"] / 1e12 if ph["device_s"] > 0 else 0.0
        if key.startswith("tcgen05"):
            ph["peak_tflops"] = pk["bf16_tflops_sustained"]
            ph["peak"] = "dense bf16 sustained, " + pk["source"]
            ph["tf32_issued_tflops"] = 3.0 * ph["tflops"]
        else:
            ph["peak_tflops"] = zpeak
            ph["peak"] = "cuBLAS complex128 GEMM 4096^3 measured on this GPU"
        ph["frac"] = ph["tflops"] / ph["peak_tflops"] if ph["peak_tflops"] else None
    rrqr_s = sum(sec for tag, n, sec, fl in table if tag.startswith("rrqr:"))
    tc = phases.get("tcgen05 split-TF32 GEMM")
    dom = tc if tc else phases.get("FP64 GEMM", {"tflops": 0.0, "peak_tflops": zpeak, "frac": None, "launches": 0})

    # the plain FP64 factorization on the same workload and refinement: one
    # warm-up and one timed step, for the mixed-vs-plain comparison
    plain = None
    info = S.info()
    if cfg.get("precision", 0) != 0 and not args.no_plain:
        from rcs_b200.solver import AIFMM
        S.close()  # the mixed solver's blocks make room for the plain one
        torch.cuda.empty_cache()
        S0 = AIFMM(K, leaf_size=cfg["leaf"], tol_pow=cfg["tol_pow"], fillin_tol=cfg["fillin_tol"],
                   n_levels=cfg["levels"], precision=0)
        S0.checkpoint()
        X0 = torch.empty_like(Bd)
        prec0 = []

        def step0():
            S0.rewind()
            S0.factorize()
            prec0.append(S0.solve_gmres_device(A, Bd.data_ptr(), nrhs, X0.data_ptr(), tol=cfg["gmres"], restart=30,
                                               maxit=300))

        step0()
        torch.cuda.synchronize()
        barrier(world)
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        step0()
        f1.record(stream)
        torch.cuda.synchronize()
        t_plain = max_over_ranks(f0.elapsed_time(f1) / 1e3, world)
        plain = {"value": t_plain, "unit": "s", "steps": 1, "warmup": 1, "gmres_iterations": prec0[-1]["iterations"],
                 "residual": sampled_residual(K, X0.cpu().numpy().T, B, nrows=512),
                 "phases_s": {k: S0.info()[k] for k in ("t_rrqr", "t_compress", "t_elim_x", "t_elim_z")},
                 "speedup_of_value": t_plain / t_step}
        S0.close()

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        cb = CPUBaseline(cfg)
        recs_cpu = [cb.sample(i, threads)[1] for i in range(3)]
        v = cb.extrapolate(recs_cpu, cb.lu_macs, cb.pair_macs)
        cpu = {"value": v, "unit": "s", "cores": threads, "kind": "port", "extrapolated": "lower bound",
               "sample": cb.describe(recs_cpu, threads)}
    if rank == 0:
        line = {
            "metric": METRIC, "value": t_step, "unit": "s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_step * 1e3, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "c128" if cfg.get("precision", 0) == 0 else "c128+tf32x3",
            "data": "synthetic",
            "config": config_block(cfg, world),
            "path": ({0: "plain complex128 factorization (reference control flow)",
                      1: "mixed factorization (split-TF32 mma.sync GEMMs)",
                      2: "mixed factorization (split-TF32 tcgen05 GEMMs)",
                      3: "mixed factorization (split-TF32 tcgen05 GEMMs, pre-tiled planes)",
                      4: "mixed factorization (split-TF32 persistent warp-specialised tcgen05 GEMMs)"}[
                         cfg.get("precision", 0)]
                     + (f", fill-ins under 1e-{cfg['drop_pow']} of their M2L block dropped"
                        if cfg.get("drop_pow") else "")
                     + (" + FP64 FGMRES" if A is not None else ", direct solve")),
            "residual": res, "residual_e2e": res_e2e, "residual_rows_sampled": min(2048, N),
            "residual_reference": "||Z x - b|| / ||b|| over seeded rows with exact FP64 matrix entries",
            "gmres": gm, "plain_fp64": plain, "assemble_s": t_asm, "operator_build_s": t_op,
            "capacitance_error": (capacitance_error(m, X[:, -1], cfg["radius"])
                                  if cfg.get("kind", "efie") == "es" else None),
            "operator_gb": (A.info()["bytes"] / 1e9) if A is not None else None,
            "factor_flops": info["flops_factor"],
            "phases_s": {k: info[k] for k in ("t_rrqr", "t_compress", "t_elim_x", "t_elim_z", "t_nonleaf")},
            "tree": {"levels": info["n_levels"], "avg_leaf": info["avg_leaf_size"], "avg_rank": info["avg_multipoles"],
                     "max_rank": info["max_rank"], "rrqr": info["n_rrqr"]},
            "gpu_launches": int(launches),
            "roofline": {"bound": "tensor",
                         "kernel": ((("zgemm_tc6_kernel" if cfg.get("precision") == 4 else "zgemm_tc5p_kernel")
                                     + " (tcgen05 split-TF32 Schur products; complex-counted 8 m n k flops per "
                                       "product)") if tc else "zgemm_grouped_kernel (FP64)"),
                         "achieved": dom["tflops"], "peak": dom["peak_tflops"], "unit": "TFLOP/s",
                         "frac": dom["frac"], "peak_source": dom.get("peak", ""),
                         "traffic": None, "launches_profiled": dom["launches"]},
            "roofline_phases": {**phases, "RRQR chains": {"device_s": rrqr_s}},
            "clocks": clk.summary(),
            "e2e": {"value": t_e2e, "unit": "s", "steps": e2e_steps, "h2d_bytes_per_step": int(16 * N * nrhs),
                    "d2h_bytes_per_step": int(16 * N * nrhs)},
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
