"""The C++ drop-in layer (include/aifmm/) builds without a GPU: its Eigen
subset computes what Eigen would on hand-checked cases, the project's drivers
compile and link against libaifmm_b200.so in both dtype modes, and the
reference's own driver (test/sphere.cpp) compiles unchanged when the reference
tree is present."""
import os
import shutil
import subprocess

import pytest

from rcs_b200 import dropin

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CPP = os.path.join(ROOT, "tests", "cpp")
# The reference source tree (vaishna77/RCS), when it is present on this machine.
REFERENCE_ROOT = os.environ.get("AIFMM_REFERENCE_ROOT", "")
REFERENCE_DRIVER = os.path.join(REFERENCE_ROOT, "test", "sphere.cpp") if REFERENCE_ROOT else ""

pytestmark = pytest.mark.skipif(shutil.which("g++") is None, reason="g++ not available")


@pytest.fixture(scope="module")
def lib():
    from rcs_b200 import build
    if shutil.which("nvcc") is None and not os.path.exists("/usr/local/cuda/bin/nvcc"):
        pytest.skip("nvcc not available")
    return build.build()


def _ok(r: subprocess.CompletedProcess) -> None:
    assert r.returncode == 0, r.stdout + r.stderr
    assert "warning" not in r.stderr, r.stderr


def test_eigen_subset_matches_hand_values(tmp_path):
    exe = str(tmp_path / "esc")
    _ok(dropin.compile_driver([os.path.join(CPP, "eigen_subset_check.cpp")], exe, link=False))
    _ok(dropin.compile_driver([os.path.join(CPP, "eigen_subset_check.cpp")], exe, extra=["-fopenmp"]))
    r = subprocess.run([exe], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0 and r.stdout.strip() == "OK", r.stdout


def test_complex_driver_links(lib, tmp_path):
    _ok(dropin.compile_driver([os.path.join(CPP, "dropin_driver.cpp")], str(tmp_path / "d")))


def test_real_mode_driver_links(lib, tmp_path):
    _ok(dropin.compile_driver([os.path.join(CPP, "dropin_es_double.cpp")], str(tmp_path / "e"),
                              defines=("USE_DOUBLE", "USE_THREE")))


@pytest.mark.skipif(not os.path.exists(REFERENCE_DRIVER), reason="reference tree not present")
def test_reference_driver_compiles_unchanged(lib, tmp_path):
    r = dropin.compile_driver([REFERENCE_DRIVER], str(tmp_path / "sphere"), extra=["-fopenmp"])
    assert r.returncode == 0, r.stderr
