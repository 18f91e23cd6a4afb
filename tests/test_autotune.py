"""Autotuner (moist_autotune, moist_batch_autotune): it leaves the State as it found it, and the
steps after it equal those of an untuned context bit for bit (every candidate computes the same
values; the choice changes only the speed)."""
import numpy as np
import pytest

from moist2d_b200 import model
from states import bubble_case, compare
from test_batch import members

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("T", [np.float32, np.float64], ids=["f32", "f64"])
def test_autotune_keeps_state_and_results(T):
    p, s = bubble_case(T, nx=96, nz=40)
    with model.Model(p) as m:
        m.upload(s)
        rep = m.autotune(2)
        back = m.download(s.copy())
        m.step(3)
        got = m.download(s.copy())
    assert "->" in rep and "strip" in rep
    compare(back, s, p, fields=("rho", "rho_u", "rho_w", "rho_theta", "rho_qv", "rho_qc", "rho_qr", "prec"))
    compare(got, model.rk3_step(s.copy(), p, 3), p)


def test_batch_autotune_keeps_state_and_results():
    mem = members(np.float32)
    with model.Ensemble([p for p, _ in mem]) as e:
        for i, (_, s) in enumerate(mem):
            e.upload(i, s)
        e.step(1)
        rep = e.autotune(2)
        e.step(2)
        got = [e.download(i, s.copy()) for i, (_, s) in enumerate(mem)]
    assert "column block" in rep
    for (p, s), g in zip(mem, got):
        compare(g, model.rk3_step(s.copy(), p, 3), p)
