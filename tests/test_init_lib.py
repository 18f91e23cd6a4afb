"""The seeded initial-state generators behind the C-ABI (moist_init_*, host code, no device)
against the numpy generators of moist2d_b200/init.py, and the discrete hydrostatic balance of
init_state! (moist.jl:413-431).

Philox4x32-10 is integer arithmetic: the library's draws equal numpy's bit for bit. The states
are built in double precision from exp / pow / tanh, whose last bits may differ between numpy's
and the C library's implementations, then rounded once to the State precision: Float64 states
agree to 1e-12 relative, Float32 states to one unit in the last place."""
import numpy as np
import pytest

from moist2d_b200 import init
from moist2d_b200.params import Params, State

FIELDS = ("rho", "rho_u", "rho_w", "rho_theta", "rho_qv", "rho_qc", "rho_qr", "prec", "theta_ref")


def _agree(a, b, T):
    for f in FIELDS:
        x, y = getattr(a, f), getattr(b, f)
        assert x.shape == y.shape and x.dtype == y.dtype, f
        if T is np.float64:
            scale = max(float(np.max(np.abs(y))), 1e-300)
            assert float(np.max(np.abs(x - y))) <= 1e-12 * scale, f
        else:
            ulps = np.abs(x.view(np.int32).astype(np.int64) - y.view(np.int32).astype(np.int64))
            assert int(np.max(ulps)) <= 1, (f, int(np.max(ulps)))


def test_uniform_draws_equal_numpy_bit_for_bit():
    idx = np.concatenate([np.arange(1000), np.array([2**32 - 1, 2**32, 2**40 + 7], dtype=np.int64)])
    for seed, stream in ((1, 0), (2, 1), (3, 1007), (0xFFFFFFFF, 5)):
        a = init.uniform_lib(seed, stream, idx)
        b = init.uniform(seed, stream, idx)
        assert np.array_equal(a, b)
        assert np.all((a > 0) & (a < 1))


@pytest.mark.parametrize("T", [np.float32, np.float64])
def test_warm_bubble(T):
    pa, a = init.warm_bubble_lib(T, seed=1, nx=40, nz=30)
    pb, b = init.warm_bubble(T, seed=1, nx=40, nz=30)
    _agree(a, b, T)
    assert float(np.max(a.rho_qv)) > 0


@pytest.mark.parametrize("T", [np.float32, np.float64])
def test_sounding_bubbles_reaching_above_12_km(T):
    # 120 levels of 125 m reach 15 km: the isothermal layer above 12 km is built too
    pa, a = init.sounding_bubbles_lib(T, nx=64, nz=120, nbub=3)
    pb, b = init.sounding_bubbles(T, nx=64, nz=120, nbub=3)
    _agree(a, b, T)


@pytest.mark.parametrize("member", [0, 1, 7])
def test_ensemble_members(member):
    pa, a = init.ensemble_member_lib(np.float32, member=member, nx_choices=(32, 48, 64), nz_choices=(20, 30))
    pb, b = init.ensemble_member(np.float32, member=member, nx_choices=(32, 48, 64), nz_choices=(20, 30))
    assert (pa.Nx, pa.Nz) == (pb.Nx, pb.Nz)
    _agree(a, b, np.float32)


@pytest.mark.parametrize("T", [np.float32, np.float64])
def test_init_state_and_its_hydrostatic_balance(T):
    """init_state! (moist.jl:351-450) on a stretched grid: the library against numpy, and the
    balance its Newton iteration solves (moist.jl:426-430): after the iteration the residual
    p_k - p_{k-1} + g (z_k - z_{k-1}) (rho_{k-1} + rho_k) / 2 is small against the pressure
    step g dz rho between the levels, with p_k = P0 (rho_k r theta_k / P0)^(cp/cv). The
    reference runs exactly ten iterations (moist.jl:413), each also relaxing qv by a factor 0.8
    towards its target, so the balance holds to ~1e-6 of the step, not to rounding."""
    p = Params(T, Nx=12, Nz=40, H=100.0 * 40 * 1.02 * 1.5, dz0=100.0, z_fact=1.05)
    a = init.init_state_lib(State(p), p, seed=3)
    b = init.init_state(State(p), p, seed=3)
    _agree(a, b, T)
    c = p.c
    Rd, Rv, Cpd, Cpv, P0, g = (float(x) for x in (c.Rd, c.Rv, c.Cpd, c.Cpv, c.P0, c.GRAV))
    cols = slice(p.is_ - 1, p.ie)
    rho = a.rho[:, cols].astype(np.float64)
    qv = a.rho_qv[:, cols] / rho
    th = a.rho_theta[:, cols] / rho
    r = Rd * (1 - qv) + Rv * qv
    cp = Cpd * (1 - qv) + Cpv * qv
    pres = P0 * (rho * r * th / P0) ** (cp / (cp - r))
    z = p.z.astype(np.float64)
    dz = np.diff(z)[:, None]
    resid = pres[1:] - pres[:-1] + g * dz * 0.5 * (rho[:-1] + rho[1:])
    step = g * dz * rho[1:]
    tol = 2e-3 if T is np.float32 else 1e-5  # Float32 states carry their rounding
    assert float(np.max(np.abs(resid) / step)) < tol
