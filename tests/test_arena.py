"""The serving layer's device-memory arena (hosono-2dmhd_b200/csrc/arena.h),
a host-only first-fit allocator, under randomised alloc/release sequences."""
import os
import shutil
import subprocess

import pytest

import pkg

CSRC = os.path.join(pkg.PKG_DIR, "csrc")
HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_arena_invariants(seed, tmp_path):
    cxx = shutil.which("g++") or shutil.which("c++")
    if not cxx:
        pytest.skip("no C++ compiler")
    exe = str(tmp_path / "arena_check")
    subprocess.run([cxx, "-std=c++17", "-O2", "-I", CSRC, os.path.join(HERE, "arena_check.cpp"), "-o", exe],
                   check=True)
    r = subprocess.run([exe, str(seed)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, (r.returncode, r.stdout, r.stderr)
