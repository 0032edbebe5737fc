"""The tensor-core GEMM autotuner (GEMM precision 5): FP32-class results like
the kernels it chooses among, one timed trial per launch class (not per
launch), choices stored in and read back from AIFMM_TUNE_FILE, and a mixed
factorization on autotuned GEMMs that FGMRES refines to 1e-8."""
import os
import subprocess
import sys

import numpy as np
import pytest

from rcs_b200 import lowrank
from rcs_b200 import mesh as M
from rcs_b200.kernel import Context, EFIEMatrix
from rcs_b200.solver import AIFMM, H2Operator

pytestmark = pytest.mark.gpu


def _mats(m, n, k, seed):
    rng = np.random.default_rng(seed)
    A = rng.standard_normal((m, k)) + 1j * rng.standard_normal((m, k))
    B = rng.standard_normal((k, n)) + 1j * rng.standard_normal((k, n))
    return A, B


def test_autotuned_gemm_accuracy_and_one_trial_per_class():
    ctx = Context(0)
    A, B = _mats(700, 500, 300, 1)
    C = lowrank.zgemm(A, B, precision=5, ctx=ctx)
    ref = A @ B
    err = np.linalg.norm(C - ref) / (np.linalg.norm(A) * np.linalg.norm(B))
    assert 1e-12 < err < 2e-6  # split TF32, not an FP64 product
    rep = ctx.tune_report()
    assert len(rep) == 1 and "tc5p" in rep[0] and "tc6" in rep[0] and "->" in rep[0]
    A2, B2 = _mats(700, 500, 300, 2)  # same class: no new trial
    lowrank.zgemm(A2, B2, precision=5, ctx=ctx)
    assert len(ctx.tune_report()) == 1
    A3, B3 = _mats(2000, 1500, 1200, 3)  # another class
    C3 = lowrank.zgemm(A3, B3, precision=5, ctx=ctx)
    assert np.linalg.norm(C3 - A3 @ B3) / (np.linalg.norm(A3) * np.linalg.norm(B3)) < 2e-6
    assert len(ctx.tune_report()) == 2
    ctx.close()


def test_tune_file_is_reused(tmp_path):
    f = tmp_path / "tune.txt"
    code = ("import numpy as np; from rcs_b200 import lowrank; from rcs_b200.kernel import Context; "
            "c = Context(0); r = np.random.default_rng(0); "
            "A = r.standard_normal((600, 400)) + 0j; B = r.standard_normal((400, 300)) + 0j; "
            "lowrank.zgemm(A, B, precision=5, ctx=c); print(len(c.tune_report()))")
    env = dict(os.environ, AIFMM_TUNE_FILE=str(f))
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    first = subprocess.run([sys.executable, "-c", code], env=env, cwd=root, capture_output=True, text=True, check=True)
    assert first.stdout.strip() == "1" and f.read_text().strip()
    second = subprocess.run([sys.executable, "-c", code], env=env, cwd=root, capture_output=True, text=True,
                            check=True)
    assert second.stdout.strip() == "0"  # the stored choice, no trial


def test_autotuned_mixed_factorization_refines():
    K = EFIEMatrix(M.icosphere(4, 0.15), 2.0e9)
    S = AIFMM(K, leaf_size=32, tol_pow=5, fillin_tol=7, n_levels=3, precision=5, drop_pow=2)
    S.factorize()
    A = H2Operator(K, leaf_size=32, tol_pow=10, n_levels=3)
    b = K.planeWaveRhs((0, 0, -1), (1, 0, 0))
    x, rec = S.solve_gmres(A, b, tol=1e-8)
    assert rec["relres"] <= 1e-8
    assert K.ctx.tune_report()  # the factorization's GEMM classes were tuned
