"""History diagnostics (moist_history_diagnostics): output_history's primitive variables
(moist.jl:1795-1835) from the device State equal the oracle's restatement bit for bit, and the
summary equals the extremes of those fields (moist.jl:1838-1843)."""
import numpy as np
import pytest

from moist2d_b200 import model
from moist2d_b200.precision import diagnostics
from oracle import bind
from states import bubble_case


def test_oracle_history_against_numpy():
    """The oracle's u, w, theta and mixing ratios against an independent numpy evaluation."""
    p, s = bubble_case(np.float64, nx=24, nz=16)
    d = bind.history_diag(s, p)
    ref = diagnostics(s.copy(), p)
    for f in ("u", "w", "theta", "qv", "qc", "qr"):
        scale = max(np.max(np.abs(ref[f])), 1e-300)
        assert np.max(np.abs(d[f] - ref[f])) <= 1e-14 * scale, f
    assert 0.0 <= d["RH"].min() and d["RH"].max() < 150.0
    assert np.all(d["thetae"] >= d["theta"] * 0.99)


@pytest.mark.gpu
@pytest.mark.parametrize("T", [np.float32, np.float64], ids=["f32", "f64"])
def test_history_diagnostics_match_oracle(T):
    p, s = bubble_case(T, nx=40, nz=24)
    with model.Model(p) as m:
        m.upload(s)
        m.step(2)
        h = m.history()
        fin = m.download(s.copy())
        part = m.history(fields=("w", "RH"))
    ref = bind.history_diag(fin, p)
    for f in bind.HISTORY_FIELDS:
        assert np.array_equal(h[f], ref[f]), f
    assert set(part) == {"w", "RH", "summary"} and np.array_equal(part["RH"], ref["RH"])
    sm = h["summary"]
    assert sm["w_min"] == float(ref["w"].min()) and sm["w_max"] == float(ref["w"].max())
    assert sm["qc_max_gkg"] == float(ref["qc"].max()) * 1000.0
    assert sm["qr_max_gkg"] == float(ref["qr"].max()) * 1000.0
    assert sm["rh_min"] == float(ref["RH"].min()) and sm["rh_max"] == float(ref["RH"].max())
