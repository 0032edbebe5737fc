"""The device sub-allocator's bookkeeping (rcs_b200/csrc/arena.cuh) under a
randomised sequence of 60,000 allocations and releases with fake chunk
addresses: ranges inside one chunk, aligned, disjoint; an emptied arena hands
every chunk back whole; adjacent chunks never merge; chunks grow 64 MB first,
then geometrically up to 512 MB a step (tests/cpp/arena_check.cpp)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(shutil.which("g++") is None, reason="g++ not available")
def test_arena_bookkeeping(tmp_path):
    exe = str(tmp_path / "arena_check")
    r = subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", os.path.join(ROOT, "tests", "cpp", "arena_check.cpp"),
                        "-o", exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    p = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert p.returncode == 0 and p.stdout.startswith("OK"), p.stdout
