"""The Riemann solver divides by shared reciprocals (SharedRecipDiv in
hosono-2dmhd_b200/csrc/physics.cuh); its quotients must be bit-identical to
IEEE division for every in-range operand pair and flag every other pair.
tests/div_check.cu runs billions of random and adversarial pairs on the GPU."""
import os
import shutil
import subprocess

import pytest

import pkg

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.gpu
@pytest.mark.parametrize("fmad", ["false", "true"])
def test_shared_reciprocal_division_matches_ieee(fmad, tmp_path):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    exe = str(tmp_path / "div_check")
    subprocess.run([nvcc, "-std=c++17", "-O3", f"--fmad={fmad}", "-gencode", "arch=compute_100a,code=sm_100a",
                    "-I", os.path.join(pkg.PKG_DIR, "csrc"), os.path.join(HERE, "div_check.cu"), "-o", exe],
                   check=True)
    r = subprocess.run([exe, str(1 << 30), "4"], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert " mismatches 0 " in r.stdout
