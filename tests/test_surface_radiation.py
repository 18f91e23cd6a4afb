"""surface_fluxes! (moist.jl:710-752) and gray_radiation! (moist.jl:776-840) as standalone entry
points (moist_surface_fluxes, moist_gray_radiation) against the oracle's restatement, bit for bit.

The State's halo columns are set apart from the periodic copies, because surface_fluxes! reads
rho_u[ks, is-1] and rho[ks, ie+1] from them; theta_ref is the State's reference profile."""
import numpy as np
import pytest

from moist2d_b200 import model
from oracle import bind

from states import small_case

SF_FIELDS = ("d_rho_u_sf", "d_rho_theta_sf", "d_rho_qv_sf", "mflux", "shflux", "lhflux")


def case(T, seed):
    p, s = small_case(T, 13, 9, seed=seed, do_sf=True, do_rd=True)
    rng = np.random.default_rng(seed)
    for f in ("rho_u", "rho"):
        a = getattr(s, f)
        a[:, :p.halo] *= (1.0 + 0.05 * rng.standard_normal((p.ka, p.halo))).astype(T)
        a[:, p.halo + p.Nx:] *= (1.0 + 0.05 * rng.standard_normal((p.ka, p.halo))).astype(T)
    if not np.any(s.theta_ref):
        s.theta_ref[:] = (s.rho_theta[:, p.halo] / s.rho[:, p.halo]).astype(T)
    return p, s


def test_oracle_surface_fluxes_read_the_halo_columns():
    """rho_u[ks, is-1] enters the wind speed of the first column (sensible and latent heat),
    rho[ks, ie+1] the momentum flux of the last column; no other column reads them."""
    p, s = case(np.float64, 3)
    c = slice(p.is_ - 1, p.ie)
    s.rho_u[0, :] = 5.0 * s.rho[0, :]  # a surface wind above uabs_min, so that uabs reads rho_u
    a, b, d = s.copy(), s.copy(), s.copy()
    b.rho_u[0, p.halo - 1] *= 1.1
    d.rho[0, p.halo + p.Nx] *= 1.1
    for x in (a, b, d):
        bind.surface_fluxes(x, p)
    assert a.shflux[c][0] != b.shflux[c][0] and a.lhflux[c][0] != b.lhflux[c][0]
    assert np.array_equal(a.shflux[c][1:], b.shflux[c][1:]) and np.array_equal(a.mflux[c], b.mflux[c])
    assert a.mflux[c][-1] != d.mflux[c][-1]
    assert np.array_equal(a.mflux[c][:-1], d.mflux[c][:-1]) and np.array_equal(a.shflux[c], d.shflux[c])


def test_oracle_gray_radiation_heats_and_cools():
    p, s = case(np.float64, 4)
    bind.gray_radiation(s, p)
    c = slice(p.is_ - 1, p.ie)
    assert np.all(np.isfinite(s.d_rho_theta_rd[:, c])) and np.any(s.d_rho_theta_rd[:, c] != 0.0)


@pytest.mark.gpu
@pytest.mark.parametrize("T", [np.float32, np.float64], ids=["f32", "f64"])
def test_surface_fluxes_match_the_oracle(T):
    p, s = case(T, 5)
    a, b = s.copy(), s.copy()
    model.surface_fluxes(a, p)
    bind.surface_fluxes(b, p)
    c = slice(p.is_ - 1, p.ie)
    for f in SF_FIELDS:
        assert np.any(getattr(b, f)[c] != 0), f
        assert np.array_equal(getattr(a, f)[c], getattr(b, f)[c]), f


@pytest.mark.gpu
@pytest.mark.parametrize("T", [np.float32, np.float64], ids=["f32", "f64"])
def test_gray_radiation_matches_the_oracle(T):
    p, s = case(T, 6)
    a, b = s.copy(), s.copy()
    model.gray_radiation(a, p)
    bind.gray_radiation(b, p)
    c = slice(p.is_ - 1, p.ie)
    assert np.any(b.d_rho_theta_rd[:, c] != 0)
    assert np.array_equal(a.d_rho_theta_rd[:, c], b.d_rho_theta_rd[:, c])
