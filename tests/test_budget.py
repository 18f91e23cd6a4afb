"""Domain budgets (moist_budget): compensated FP64 sums of mass, water (air + fallen rain),
total energy (the kinetic, potential and internal energy densities of output_history,
moist.jl:1797-1841, times the cell volume dx dz) and accumulated rain. The oracle forms the
same per-cell terms on the CPU; their exactly rounded sum (math.fsum) is the reference for the
device's compensated sum."""
import math

import numpy as np
import pytest

from moist2d_b200 import model
from oracle import bind as ob
from states import bubble_case, small_case


def exact_budget(s, p):
    mass, water, energy, rain = ob.budget_terms(s, p)
    r = math.fsum(rain.ravel())
    return np.array([math.fsum(mass.ravel()), math.fsum(list(water.ravel()) + list(rain)),
                     math.fsum(energy.ravel()), r])


@pytest.mark.parametrize("T", [np.float32, np.float64], ids=["f32", "f64"])
def test_oracle_budget_terms(T):
    """Mass and water terms are the cell values times dz dx in double precision; the energy is
    dominated by the internal energy and positive; the water sum includes the rain."""
    p, s = bubble_case(T, nx=24, nz=16)
    s.prec[p.is_ - 1:p.ie] = np.linspace(0.0, 1e-3, p.Nx).astype(T)
    mass, water, energy, rain = ob.budget_terms(s, p)
    cols = slice(p.is_ - 1, p.ie)
    vol = p.dz.astype(np.float64)[:, None] * float(p.dx)
    np.testing.assert_array_equal(mass, s.rho[:, cols].astype(np.float64) * vol)
    wsum = (s.rho_qv[:, cols].astype(np.float64) + s.rho_qc[:, cols].astype(np.float64)
            + s.rho_qr[:, cols].astype(np.float64))
    np.testing.assert_array_equal(water, wsum * vol)
    np.testing.assert_array_equal(rain, s.prec[cols].astype(np.float64) * float(p.dx))
    assert np.all(energy > 0)
    b = exact_budget(s, p)
    assert b[1] > math.fsum(water.ravel()) and b[3] == math.fsum(rain)


@pytest.mark.gpu
@pytest.mark.parametrize("T", [np.float32, np.float64], ids=["f32", "f64"])
@pytest.mark.parametrize("case", ["bubble", "small"])
def test_gpu_budget_matches_exact_sum(T, case):
    """The device's compensated sums agree with the exactly rounded sums of the oracle's terms
    to a few units in the last place, after steps that create rain, and are reproducible."""
    p, s = bubble_case(T, nx=96, nz=40) if case == "bubble" else small_case(T, 37, 11)
    with model.Model(p) as m:
        m.upload(s)
        m.step(3)
        got = m.budget()
        again = m.budget()
        m.download(s)
    ref = exact_budget(s, p)
    np.testing.assert_array_equal(got, again)
    np.testing.assert_allclose(got, ref, rtol=1e-14, atol=0)
    assert ref[3] >= 0
