"""The Float32 error statement tool (moist2d_b200.precision) on the host: its comparison and its
report of a run that stops at a NaN, with a stand-in for the device Model."""
import numpy as np

from moist2d_b200 import model, precision

from states import bubble_case


class FakeModel:
    """Steps nothing; raises FloatingPointError at a chosen step per precision."""
    nan_at = {}

    def __init__(self, p, flags=0):
        self.p, self.n = p, 0

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        return False

    def upload(self, s):
        pass

    def step(self, k):
        self.n += k
        if self.n == self.nan_at.get(np.dtype(self.p.T).name):
            raise FloatingPointError("NaN detected in rho")

    def download(self, s):
        pass


def builder(T):
    return bubble_case(T, nx=8, nz=6)


def test_precision_reports_the_step_of_a_nan(monkeypatch):
    monkeypatch.setattr(model, "Model", FakeModel)
    monkeypatch.setattr(FakeModel, "nan_at", {"float32": 5, "float64": 7})
    out = precision.run(builder, 10)
    assert out == {"nan": {"float32": {"step": 5, "error": "NaN detected in rho"},
                           "float64": {"step": 7, "error": "NaN detected in rho"}}}


def test_precision_compares_runs_that_finish(monkeypatch):
    """Without a NaN the two precisions are compared field by field; the stand-in leaves both
    at their initial states, which differ only by the Float32 rounding of the start."""
    monkeypatch.setattr(model, "Model", FakeModel)
    monkeypatch.setattr(FakeModel, "nan_at", {})
    out = precision.run(builder, 3)
    assert set(out) == set(precision.FIELDS)
    for f in ("theta", "qv"):
        assert 0.0 < out[f]["rel_l2"] < 1e-6, (f, out[f])


def test_control_run_starts_one_ulp_away(monkeypatch):
    """--control: the first run is Float64 from a start whose rho_theta differs from the other's
    by exactly one ulp in every interior cell (the stand-in steps nothing, so the comparison sees
    the start itself)."""
    p, s = bubble_case(np.float64, nx=8, nz=6)
    t = s.copy()
    precision.last_bit_perturbed(t, p)
    c = slice(p.is_ - 1, p.ie)
    a, b = s.rho_theta[:, c], t.rho_theta[:, c]
    ulps = np.abs(a.view(np.int64) - b.view(np.int64))
    assert np.all(ulps == 1)
    assert 0 < np.mean(b > a) < 1  # both directions occur
    monkeypatch.setattr(model, "Model", FakeModel)
    monkeypatch.setattr(FakeModel, "nan_at", {})
    out = precision.run(lambda T: bubble_case(T, nx=8, nz=6), 3, control=True)
    assert 0.0 < out["theta"]["rel_l2"] < 1e-15
    assert out["qv"]["rel_l2"] == 0.0
