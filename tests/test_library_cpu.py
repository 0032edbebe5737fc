"""CPU-side checks of the CUDA library: it builds for sm_100a, loads, and
exports exactly the entry points that include/*.h declares (no GPU calls)."""
import glob
import os
import re
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions() -> set[str]:
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(aifmm_\w+)\s*\(", src, flags=re.M):
            names.add(m.group(1))
    return names


@pytest.fixture(scope="module")
def libpath():
    from rcs_b200 import build
    if shutil.which("nvcc") is None and not os.path.exists("/usr/local/cuda/bin/nvcc"):
        pytest.skip("nvcc not available")
    return build.build()


def test_header_declares_entry_points():
    names = declared_functions()
    assert "aifmm_ctx_create" in names and "aifmm_kernel_matrix" in names
    assert len(names) >= 15


def test_library_exports_every_declared_symbol(libpath):
    out = subprocess.run(["nm", "-D", "--defined-only", libpath], capture_output=True, text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    missing = declared_functions() - exported
    assert not missing, f"declared but not exported: {sorted(missing)}"


def test_python_binding_covers_header(libpath):
    from rcs_b200 import _lib
    assert declared_functions() == set(_lib.exported_symbols())
    L = _lib.lib()  # loads the .so and resolves every symbol
    assert L is not None


def test_build_targets_sm100a_only():
    from rcs_b200 import build
    assert build.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]
