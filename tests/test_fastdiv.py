"""Markstein division (moist2d_b200/csrc/fastdiv.cuh) equals IEEE division bit for bit for every
finite numerator in its unflagged range, for the denominators the tracer sweep divides by
(dx, dz, dz sums, z differences, 3, densities) and for random denominators in [2^-20, 2^20]."""
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


def test_markstein_division_is_ieee_exhaustively(tmp_path):
    exe = tmp_path / "fastdiv_check"
    subprocess.run(["nvcc", "-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a",
                    "--fmad=false", "-o", str(exe), os.path.join(HERE, "fastdiv_check.cu")], check=True)
    rng = np.random.default_rng(7)
    model_b = [250.0, 125.0, 100.0, 375.0, 250.0 + 250.0, 3.0, 1.1535, 0.8123, 0.3141, 62.5, 102.5]
    rand_b = list(np.float32(2.0) ** rng.uniform(-20, 20, 12)) + list(rng.uniform(0.05, 1.4, 6))
    bs = [repr(float(np.float32(b))) for b in model_b + rand_b]
    out = subprocess.run([str(exe)] + bs, capture_output=True, text=True, timeout=600)
    lines = [l.split() for l in out.stdout.strip().splitlines()]
    assert len(lines) == len(bs), out.stdout + out.stderr
    for b, mism, flagged in lines:
        assert int(mism) == 0, "denominator %s: %s mismatches" % (b, mism)
    assert out.returncode == 0
