"""The OpenMP build of the oracle (the timed CPU baseline, oracle/libmoist_oracle_omp.so)
against the single-thread parity oracle.

The OpenMP build restates the reference's Threads.@threads tracer sweep: each thread sweeps a
contiguous chunk of columns in order and reads the two columns left of its chunk at their
pre-sweep values. With one thread that is the serial lexicographic sweep, so the two builds
must agree bit for bit; with several threads the result depends on the chunking (as the
threaded reference's does), so the build is used for timing only."""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SCRIPT = r"""
import ctypes as C, sys
import numpy as np
sys.path.insert(0, sys.argv[1]); sys.path.insert(0, sys.argv[1] + '/tests')
from oracle import bind
from states import bubble_case
Ls = bind.lib()
Lo = C.CDLL(sys.argv[1] + '/oracle/libmoist_oracle_omp.so')
Lo.oracle_rk3_step.argtypes = Ls.oracle_rk3_step.argtypes
bad = []
for T in (np.float64, np.float32):
    p, s1 = bubble_case(T, nx=40, nz=16)
    s2 = s1.copy()
    cp = p.to_c(); h1 = s1.to_c(); h2 = s2.to_c()
    assert Ls.oracle_rk3_step(C.byref(cp), p.precision, 1, C.byref(h1), 6) == -1
    assert Lo.oracle_rk3_step(C.byref(cp), p.precision, 1, C.byref(h2), 6) == -1
    bad += [T.__name__ + ':' + f for f in ('rho', 'rho_u', 'rho_w', 'rho_theta', 'rho_qv', 'rho_qc', 'rho_qr', 'prec')
            if not np.array_equal(getattr(s1, f), getattr(s2, f))]
print(','.join(bad))
"""


def _differing(threads):
    so = os.path.join(ROOT, "oracle", "libmoist_oracle_omp.so")
    if not os.path.exists(so):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)
    env = dict(os.environ, OMP_NUM_THREADS=str(threads))
    out = subprocess.run([sys.executable, "-c", SCRIPT, ROOT], env=env, capture_output=True, text=True,
                         timeout=300)
    assert out.returncode == 0, out.stderr
    return [x for x in out.stdout.strip().split(",") if x]


def test_omp_oracle_one_thread_is_the_serial_oracle():
    assert _differing(1) == []


def test_omp_oracle_threads_change_only_the_sweep_seams():
    """With 4 threads the chunk seams of the tracer sweep read pre-sweep values: the tracers
    (and through them the rest of the State) differ from the serial sweep."""
    d = _differing(4)
    assert any(x.endswith("rho_qv") for x in d), d
