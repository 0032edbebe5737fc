"""bench.py's reference arm and CPU baseline on the CPU: the reference's
algorithm (the oracle) timed on bounded samples of the workload's own tree,
extrapolated to the workload as a lower bound, with no GPU library loaded;
the arm's `config` is the GPU arm's, so the two lines pair up; and the
extrapolation is below the oracle's full factor+solve where that can be run
(N = 1,920)."""
import json
import os
import subprocess
import sys
import time

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def test_reference_arm_line_and_no_gpu_library():
    code = (
        "import sys, json; sys.path.insert(0, %r); sys.argv = ['bench.py', '--impl', 'reference', '--config', 'c1', "
        "'--steps', '2', '--warmup', '1']; import bench; bench.main(); "
        "maps = open('/proc/self/maps').read(); print(json.dumps({'gpu_lib': 'libaifmm_b200' in maps}))" % ROOT)
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    lines = [json.loads(x) for x in r.stdout.strip().splitlines()]
    line, probe = lines[0], lines[1]
    assert probe["gpu_lib"] is False
    import bench
    assert line["impl"] == "reference" and line["warmup"] == 1 and line["steps"] == 2
    assert line["config"] == bench.config_block(bench.CONFIGS["c1"], 1)
    assert line["extrapolated"] == "lower bound" and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] >= 1
    assert line["single_thread"]["cores"] == 1 and line["single_thread"]["value"] > 0
    assert len(line["samples"]) == 2


def test_lower_bound_is_below_full_oracle_run():
    """At N = 1,920 (config 1) the oracle's whole factor + solve runs in
    seconds on one thread; the sampled extrapolation must not exceed it."""
    import bench
    import oracle
    from rcs_b200 import mesh as M
    cfg = bench.CONFIGS["c1"]
    K = oracle.EFIE(M.icosphere(cfg["sub"], cfg["radius"]), cfg["freq"])
    b = K.rhs_plane((0, 0, -1), (1, 0, 0))
    oracle.set_threads(1)
    try:
        S = oracle.AIFMM(K, leaf_size=cfg["leaf"], tol_pow=cfg["tol_pow"], fillin_tol=cfg["fillin_tol"])
        t0 = time.perf_counter()
        S.factorize()
        S.solve(b)
        full = time.perf_counter() - t0
    finally:
        oracle.set_threads(os.cpu_count() or 1)
    cb = bench.CPUBaseline(cfg)
    recs = [cb.sample(i, 1)[1] for i in range(3)]
    bound = cb.extrapolate(recs, cb.lu_macs, cb.pair_macs)
    assert 0 < bound < full
    # the model counts exactly the near-field updates of the elimination order
    sizes = np.array([len(v) for v in cb.leaves])
    assert sizes.sum() == K.N
