"""The branch-free divisions of the tracer sweep (moist2d_b200/csrc/fastdiv.cuh) equal CUDA's IEEE
division bit for bit, for every numerator with the denominators the model divides by (and ones
that make exact ties in the subnormal range) and on random bit patterns of every class:
FP64-reciprocal division wherever its subnormal guard lets the quotient through, its explicit
subnormal-rounding form everywhere. Also the PTX min / max against Julia's semantics."""
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def checker(tmp_path_factory):
    exe = tmp_path_factory.mktemp("fastdiv") / "fastdiv_check"
    subprocess.run(["nvcc", "-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a",
                    "--fmad=false", "-o", str(exe), os.path.join(HERE, "fastdiv_check.cu")], check=True)
    return str(exe)


def run(checker, *args, timeout=600):
    out = subprocess.run([checker] + [str(a) for a in args], capture_output=True, text=True, timeout=timeout)
    assert out.returncode in (0, 1), out.stdout + out.stderr
    return [line.split() for line in out.stdout.strip().splitlines()]


def test_div64_every_numerator(checker):
    rng = np.random.default_rng(7)
    model_b = [250.0, 125.0, 100.0, 375.0, 500.0, 3.0, 1.1535, 0.8123, 0.3141, 62.5, 102.5, 1.0]
    special = [1e-45, -3e-39, 1.17549435e-38, 3.4028235e38, -7.0, 2.0 ** -126, 2.0 ** 127, 6.0, 10.0, -12.0]
    rand_b = list(np.float32(2.0) ** rng.uniform(-60, 60, 8)) + list(-rng.uniform(0.05, 1.4, 4))
    bs = [repr(float(np.float32(b))) for b in model_b + special + rand_b]
    lines = run(checker, "div64", *bs)
    assert len(lines) == len(bs)
    for b, mv, mc, guarded, mxv, mxc in lines:
        assert (int(mv), int(mc), int(mxv), int(mxc)) == (0, 0, 0, 0), "denominator %s: %s" % (b, (mv, mc, mxv, mxc))


def test_div64_random_bit_patterns(checker):
    ((_, mv, mc, guarded, mxv, mxc, skipped),) = run(checker, "random", 1 << 32, 11)
    assert (int(mv), int(mc), int(mxv), int(mxc)) == (0, 0, 0, 0)
    assert int(skipped) < (1 << 32) // 100


def test_rcp64_accuracy(checker):
    # the proof needs |1 - b y| well below 2^-49; rcp64 reaches a few units of 2^-53
    ((_, worst),) = run(checker, "rcp64")
    assert float(worst) < 4.0


def test_julia_min_max(checker):
    assert run(checker, "minmax") == [["minmax", "0"]]
