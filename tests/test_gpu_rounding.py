"""The push's own reciprocal and square root (spectral_rs_b200/csrc/exact_math.cuh) against
the IEEE round-to-nearest operations: every float in [1, 2^126), and the guarded versions on
special values.  The particle kernels are bit-exact with the reference only if these agree
everywhere on the domain the push uses."""
import os
import subprocess

import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu


def test_exact_math_matches_ieee_on_its_domain(tmp_path):
    exe = tmp_path / "rounding_check"
    subprocess.run(["/usr/local/cuda/bin/nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-O3",
                    "-I", os.path.join(ROOT, "spectral_rs_b200", "csrc"), os.path.join(ROOT, "tests", "rounding_check.cu"),
                    "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    print("\n" + r.stdout.strip())
    assert r.returncode == 0, r.stdout + r.stderr
