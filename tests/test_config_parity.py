"""GPU parity on the benchmark workloads at their full sizes, bit for bit against the serial
oracle (rk3_step!, moist.jl:1589-1683, with the in-place Gauss-Seidel tracer sweep of
moist.jl:1469-1518 in its single-thread order).

- warm moist bubble, 200 x 100 cells of 100 m, ns = 6 (stage substeps 2, 3, 6), dt = 1 s:
  300 large steps in each precision mode, and 1800 steps (the whole run) in Float64;
- sounding with a row of five bubbles, 2048 x 128 cells of 250 m x 125 m, ns = 8 (3, 4, 8),
  dt = 2 s: 10 large steps with the strip width and tracer sweep the autotuner picks (what
  the benchmark runs), with the row-streaming sweep, and in Float64.

Every interior cell of the seven prognostic fields and the accumulated rain must be equal.
The oracle runs single-threaded: about 20 s per 300 warm-bubble steps, 0.8 s per sounding
step on one core."""
import numpy as np
import pytest

from moist2d_b200 import abi, model
from moist2d_b200.init import sounding_bubbles, warm_bubble
from oracle import bind

from states import compare

pytestmark = pytest.mark.gpu

MODES = [(np.float32, False), (np.float32, True), (np.float64, False)]
MODE_IDS = ["f32-tri64", "f32-tri32", "f64"]


def _flags(tri_native):
    return abi.MOIST_FLAG_TRI_NATIVE if tri_native else 0


def _tri64(T, tri_native):
    return T is np.float64 or not tri_native


def _active(s, p):
    """The case must exercise the Kessler branches: cloud water and rain present."""
    is0, ie0 = p.is_ - 1, p.ie
    return float(np.max(s.rho_qc[:, is0:ie0])) > 0 and float(np.max(s.rho_qr[:, is0:ie0])) > 0


@pytest.mark.parametrize("T,tri_native", MODES, ids=MODE_IDS)
def test_warm_bubble_full_size_300_steps(T, tri_native):
    p, s = warm_bubble(T)
    assert (p.Nx, p.Nz, p.ns, float(p.dt)) == (200, 100, 6, 1.0)
    a, b = s.copy(), s.copy()
    model.rk3_step(a, p, 300, flags=_flags(tri_native))
    bind.rk3_step(b, p, 300, tri64=_tri64(T, tri_native))
    compare(a, b, p)
    assert _active(b, p)


def test_warm_bubble_full_size_1800_steps_f64():
    p, s = warm_bubble(np.float64)
    a, b = s.copy(), s.copy()
    model.rk3_step(a, p, 1800)
    bind.rk3_step(b, p, 1800, tri64=True)
    compare(a, b, p)
    assert float(np.max(b.prec)) > 0  # rain has reached the ground


@pytest.fixture(scope="module")
def sounding_oracle():
    """The oracle's 10 steps of the 2048 x 128 sounding workload in Float32 (FP64 elimination),
    shared by the Float32 variants below."""
    p, s = sounding_bubbles(np.float32)
    b = s.copy()
    bind.rk3_step(b, p, 10, tri64=True)
    return p, s, b


def test_sounding_full_size_autotuned(sounding_oracle):
    """The benchmark's configuration: autotuned strip width and tracer sweep."""
    p, s, b = sounding_oracle
    assert (p.Nx, p.Nz, p.ns, float(p.dt)) == (2048, 128, 8, 2.0)
    a = s.copy()
    with model.Model(p) as m:
        m.upload(s)
        report = m.autotune(2)  # restores the State it tuned on
        m.step(10)
        m.download(a)
    assert " -> strip " in report
    compare(a, b, p)


def test_sounding_full_size_default_stream_and_dataflow(sounding_oracle):
    p, s, b = sounding_oracle
    for flags in (0, abi.MOIST_FLAG_TRACER_STREAM, abi.MOIST_FLAG_TRACER_DATAFLOW):
        a = s.copy()
        model.rk3_step(a, p, 10, flags=flags)
        compare(a, b, p)


def test_sounding_full_size_f64():
    p, s = sounding_bubbles(np.float64)
    a, b = s.copy(), s.copy()
    model.rk3_step(a, p, 6)
    bind.rk3_step(b, p, 6, tri64=True)
    compare(a, b, p)
