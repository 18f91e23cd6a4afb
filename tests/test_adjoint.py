"""Adjoint of the large step (moist_adjoint_run) against central finite differences.

The objective is the one of the adjoint workload: accumulated surface rain sum(prec * dx)
after n large steps, plus (in the first test) seeded weights on every prognostic field of the
final State, so that every path of the step carries gradient. Directional derivatives of the
adjoint, <grad, v>, are compared with central differences (J(x + h v) - J(x - h v)) / 2h of the
oracle's Float64 step (the CPU restatement, bitwise equal to the library's Float64 step) on
seeded random directions v in the seven prognostic fields and in K_auto and Qc_threshold.
The step is piecewise smooth (upwind and limiter switches, Kessler clamps), so the directions
are scaled to stay well inside the pieces: h = 1e-6 relative to each field's magnitude (1e-4
for the two parameters, whose effect on J is small enough that a smaller step loses digits to
rounding).

The same gradients are also compared with the exact directional derivative of the oracle's
Float64 step computed in forward mode with dual numbers (bind.tangent, oracle_tangent.cpp: the
ForwardDiff-style derivative of the restated step), where no truncation error hides a
discrepancy."""
import numpy as np
import pytest

from moist2d_b200 import abi, model
from moist2d_b200.init import single_bubble
from moist2d_b200.params import Constants
from oracle import bind

from states import bubble_case

pytestmark = pytest.mark.gpu

FIELDS = abi.PROGNOSTIC


def _interior(p):
    return slice(p.is_ - 1, p.ie)


def objective(s, p, prec_w, seeds):
    """J = sum(prec_w * prec) + sum_f sum(seeds[f] * S.f), halo columns excluded."""
    c = _interior(p)
    J = float(np.sum(prec_w[c] * s.prec[c].astype(np.float64)))
    for f, w in seeds.items():
        J += float(np.sum(w[:, c] * getattr(s, f)[:, c].astype(np.float64)))
    return J


def oracle_J(p, s, nsteps, prec_w, seeds):
    a = s.copy()
    bind.rk3_step(a, p, nsteps, tri64=True)
    return objective(a, p, prec_w, seeds)


def direction(p, s, rng, fields=FIELDS):
    """Random perturbation of the interior, each field scaled by its own magnitude (tracers by
    their local value, so that cells without cloud or rain stay without)."""
    c = _interior(p)
    v = {}
    for f in fields:
        x = getattr(s, f).astype(np.float64)
        d = np.zeros_like(x)
        if f in ("rho_qv", "rho_qc", "rho_qr"):
            d[:, c] = x[:, c] * rng.standard_normal(x[:, c].shape)
        else:
            d[:, c] = np.max(np.abs(x[:, c])) * rng.standard_normal(x[:, c].shape)
        if f == "rho_w":
            d[-1, :] = 0.0  # the lid stays 0
        v[f] = d
    return v


def shifted(s, v, h):
    a = s.copy()
    for f, d in v.items():
        x = getattr(a, f)
        x[...] = (x.astype(np.float64) + h * d).astype(x.dtype)
    return a


def with_constants(p, **kw):
    c = {k: getattr(p.c, k) for k in ("K_auto", "Qc_threshold")}
    c.update(kw)
    return p.replace(constants=Constants(p.T, **{k: float(x) for k, x in c.items()}))


def fd_check(p, s, nsteps, prec_w, seeds, grads, ndir, seed, h=1e-6, hpar=1e-4, rtol=5e-4):
    rng = np.random.default_rng(seed)
    worst = 0.0
    for _ in range(ndir):
        v = direction(p, s, rng)
        ad = sum(float(np.sum(grads[f] * v[f])) for f in FIELDS)
        fd = (oracle_J(p, shifted(s, v, h), nsteps, prec_w, seeds)
              - oracle_J(p, shifted(s, v, -h), nsteps, prec_w, seeds)) / (2 * h)
        err = abs(ad - fd) / max(abs(fd), 1e-300)
        worst = max(worst, err)
        assert err <= rtol, "state direction: adjoint %.10e vs central difference %.10e (rel %.2e)" % (ad, fd, err)
    for name in ("K_auto", "Qc_threshold"):
        x0 = float(getattr(p.c, name))
        hp = hpar * x0
        fd = (oracle_J(with_constants(p, **{name: x0 + hp}), s, nsteps, prec_w, seeds)
              - oracle_J(with_constants(p, **{name: x0 - hp}), s, nsteps, prec_w, seeds)) / (2 * hp)
        ad = grads["k_auto" if name == "K_auto" else "qc_threshold"]
        err = abs(ad - fd) / max(abs(fd), 1e-300)
        worst = max(worst, err)
        assert err <= rtol, "%s: adjoint %.10e vs central difference %.10e (rel %.2e)" % (name, ad, fd, err)
    return worst


def rain_weight(p):
    w = np.zeros(p.ia)
    w[_interior(p)] = float(p.dx)
    return w


def state_seeds(p, s, seed):
    """Seeded weights on the final State, each field normalised by its magnitude."""
    rng = np.random.default_rng(seed)
    c = _interior(p)
    out = {}
    for f in FIELDS:
        x = getattr(s, f).astype(np.float64)
        w = np.zeros_like(x)
        w[:, c] = rng.standard_normal(x[:, c].shape) / max(np.max(np.abs(x[:, c])), 1e-30) / x[:, c].size
        out[f] = w
    return out


def run_adjoint(p, s, nsteps, ckpt, prec_w, seeds, flags=0, tapes=-1):
    with model.Model(p, flags) as m:
        m.upload(s)
        m.set_adjoint_tapes(tapes)
        g = m.adjoint(nsteps, ckpt, prec_weight=prec_w, state_seed=seeds)
        fin = s.copy()
        m.download(fin)
    return g, fin


@pytest.mark.parametrize("nsteps", [1, 4])
def test_adjoint_matches_central_differences_f64(nsteps):
    p, s = bubble_case(np.float64, nx=24, nz=16)
    prec_w = rain_weight(p)
    seeds = state_seeds(p, s, 11)
    g, _ = run_adjoint(p, s, nsteps, 2, prec_w, seeds)
    assert np.isclose(g["objective"], oracle_J(p, s, nsteps, prec_w, seeds), rtol=1e-13, atol=0.0)
    fd_check(p, s, nsteps, prec_w, seeds, g, ndir=4, seed=nsteps)


def test_adjoint_rain_objective_f64():
    """The rain objective alone, after enough steps for sedimentation to reach the ground."""
    p, s = bubble_case(np.float64, nx=32, nz=20)
    prec_w = rain_weight(p)
    g, _ = run_adjoint(p, s, 12, 5, prec_w, {})
    assert g["objective"] > 0.0
    fd_check(p, s, 12, prec_w, {}, g, ndir=3, seed=5, rtol=1e-3)


def test_adjoint_checkpoint_interval_and_tape_mode_invariance():
    """The gradient does not depend on the checkpoint interval or on the tape mode (a tape per
    step of a segment, or one tape and the segment's States)."""
    p, s = bubble_case(np.float64, nx=24, nz=16)
    prec_w = rain_weight(p)
    seeds = state_seeds(p, s, 3)
    ref, _ = run_adjoint(p, s, 6, 6, prec_w, seeds, tapes=1)
    for ck, tapes in ((1, 1), (4, 1), (4, 0), (6, 0)):
        g, _ = run_adjoint(p, s, 6, ck, prec_w, seeds, tapes=tapes)
        for f in FIELDS:
            scale = np.max(np.abs(ref[f]))
            assert np.max(np.abs(g[f] - ref[f])) <= 1e-12 * scale, f
        assert np.isclose(g["k_auto"], ref["k_auto"], rtol=1e-12)


@pytest.mark.parametrize("T", [np.float32, np.float64], ids=["f32", "f64"])
def test_adjoint_leaves_the_forward_final_state(T):
    p, s = bubble_case(T, nx=24, nz=16)
    g, fin = run_adjoint(p, s, 5, 2, rain_weight(p), {})
    ref = s.copy()
    model.rk3_step(ref, p, 5)
    c = _interior(p)
    for f in FIELDS + ("prec",):
        x, y = getattr(fin, f), getattr(ref, f)
        x = x[..., c] if x.ndim == 2 else x[c]
        y = y[..., c] if y.ndim == 2 else y[c]
        assert np.array_equal(x, y), f


def test_adjoint_f32_against_f64():
    """Float32 trajectory with the double adjoint against the Float64 run: stated agreement of
    the gradient fields and the parameter gradients."""
    p64, s64 = bubble_case(np.float64, nx=32, nz=20)
    p32, s32 = bubble_case(np.float32, nx=32, nz=20)
    g64, _ = run_adjoint(p64, s64, 8, 4, rain_weight(p64), {})
    g32, _ = run_adjoint(p32, s32, 8, 4, rain_weight(p32), {})
    for f in FIELDS:
        nb = np.linalg.norm(g64[f])
        assert np.linalg.norm(g32[f] - g64[f]) <= 2e-2 * nb, f
    for k in ("k_auto", "qc_threshold"):
        assert abs(g32[k] - g64[k]) <= 2e-2 * abs(g64[k]), k


def test_adjoint_rejects_surface_fluxes():
    p, s = bubble_case(np.float64, nx=24, nz=16)
    p = p.replace(do_sf=True)
    with model.Model(p) as m:
        m.upload(s)
        with pytest.raises(NotImplementedError):
            m.adjoint(1, 1, prec_weight=rain_weight(p))


def test_adjoint_single_bubble_short():
    """The adjoint workload's domain (512 x 96, one 2 K bubble on the analytic sounding), a short
    window, rain objective plus a state seed; FD on two directions through the oracle."""
    p, s = single_bubble(np.float64)
    prec_w = rain_weight(p)
    seeds = state_seeds(p, s, 9)
    g, _ = run_adjoint(p, s, 3, 2, prec_w, seeds)
    fd_check(p, s, 3, prec_w, seeds, g, ndir=2, seed=21)


@pytest.mark.parametrize("nx,nz", [(2, 2), (3, 5), (5, 3)])
def test_adjoint_tiny_shapes(nx, nz):
    """Shapes where the periodic wraps alias (i-2 = i+1 for nx = 3, all reads one column for
    nx = 2), the linear-index clamp reads column 0, and the w-p system has one unknown."""
    from states import small_case
    p, s = small_case(np.float64, nx, nz, do_sf=False, do_rd=False)
    prec_w = rain_weight(p)
    seeds = state_seeds(p, s, 13)
    g, _ = run_adjoint(p, s, 2, 1, prec_w, seeds)
    assert np.isclose(g["objective"], oracle_J(p, s, 2, prec_w, seeds), rtol=1e-13, atol=0.0)
    fd_check(p, s, 2, prec_w, seeds, g, ndir=3, seed=nx * 10 + nz, h=1e-7)


def tangent_check(p, s, nsteps, prec_w, seeds, g, ndir, seed, rtol=1e-12):
    """<grad, v> against the exact directional derivative of the oracle's Float64 step (forward
    mode, dual numbers: oracle_tangent.cpp), in seeded state directions and in the two
    parameters. No truncation error on either side, so the tolerance is rounding only; the
    state error is taken relative to sum |grad * v| (the size of the terms that cancel)."""
    rng = np.random.default_rng(seed)
    worst = 0.0
    for _ in range(ndir):
        v = direction(p, s, rng)
        ad = sum(float(np.sum(g[f] * v[f])) for f in FIELDS)
        scale = sum(float(np.sum(np.abs(g[f] * v[f]))) for f in FIELDS)
        J, dJ = bind.tangent(p, s, nsteps, direction=v, prec_weight=prec_w, state_weight=seeds)
        assert np.isclose(J, g["objective"], rtol=1e-13, atol=0.0)
        assert scale > 0.0
        err = abs(ad - dJ) / scale
        worst = max(worst, err)
        assert err <= rtol, "adjoint %.15e vs forward mode %.15e (rel %.2e)" % (ad, dJ, err)
    for key, kw in (("k_auto", "d_k_auto"), ("qc_threshold", "d_qc_threshold")):
        _, dJ = bind.tangent(p, s, nsteps, prec_weight=prec_w, state_weight=seeds, **{kw: 1.0})
        err = abs(g[key] - dJ) / max(abs(dJ), 1e-300)
        worst = max(worst, err)
        assert err <= rtol, "%s: adjoint %.15e vs forward mode %.15e (rel %.2e)" % (key, g[key], dJ, err)
    return worst


@pytest.mark.parametrize("nsteps", [1, 4, 20])
def test_adjoint_matches_forward_mode_oracle(nsteps):
    p, s = bubble_case(np.float64, nx=24, nz=16)
    prec_w = rain_weight(p)
    seeds = state_seeds(p, s, 11)
    g, _ = run_adjoint(p, s, nsteps, 3, prec_w, seeds)
    tangent_check(p, s, nsteps, prec_w, seeds, g, ndir=4, seed=100 + nsteps)


def test_adjoint_matches_forward_mode_oracle_single_bubble():
    """The adjoint workload's domain (512 x 96), rain objective plus a state seed, 10 steps."""
    p, s = single_bubble(np.float64)
    prec_w = rain_weight(p)
    seeds = state_seeds(p, s, 9)
    g, _ = run_adjoint(p, s, 10, 5, prec_w, seeds)
    tangent_check(p, s, 10, prec_w, seeds, g, ndir=2, seed=7)


@pytest.mark.parametrize("nx,nz", [(2, 2), (3, 5), (5, 3)])
def test_adjoint_tiny_shapes_forward_mode(nx, nz):
    from states import small_case
    p, s = small_case(np.float64, nx, nz, do_sf=False, do_rd=False)
    prec_w = rain_weight(p)
    seeds = state_seeds(p, s, 13)
    g, _ = run_adjoint(p, s, 3, 2, prec_w, seeds)
    tangent_check(p, s, 3, prec_w, seeds, g, ndir=3, seed=nx * 10 + nz)


FIXTURE_RTOL = 1e-12


def fixture_errors(fx, p, s, g):
    """Relative differences of the adjoint from the fixture's forward-mode derivatives: per
    direction |<grad, v> - dJ| / sum |grad * v|, per parameter |g - dJ| / |dJ|."""
    from moist2d_b200.adjoint_check import controls, directions
    cg = controls(p, s, g)
    errs = []
    for (d_th, d_qv), ref in zip(directions(fx["seed"], fx["dirs"], p.Nz, p.Nx), fx["directions"]):
        assert np.isclose(float(np.sum(d_th * d_th)), ref["norm2_theta"], rtol=1e-12, atol=0.0)
        assert np.isclose(float(np.sum(d_qv * d_qv)), ref["norm2_qv"], rtol=1e-12, atol=0.0)
        ad = float(np.sum(cg["theta"] * d_th) + np.sum(cg["qv"] * d_qv))
        scale = float(np.sum(np.abs(cg["theta"] * d_th)) + np.sum(np.abs(cg["qv"] * d_qv)))
        errs.append(abs(ad - ref["dJ"]) / scale)
    par = {k: abs(g[k] - v) / abs(v) for k, v in fx["params"].items()}
    return errs, par


def test_adjoint_single_bubble_matches_forward_mode_fixture():
    """The adjoint workload (512 x 96 single bubble, Float64, rain objective) over the configured
    600 steps against the exact directional derivatives of the oracle's step in forward mode
    (tests/golden/tangent_single_bubble.json, made by tests/golden/make_tangent_single_bubble.py):
    <grad, v> in 16 seeded large-scale directions of theta' and qv, and both parameter gradients.
    Central differences cannot serve here (over 600 steps they scatter on some directions); the
    forward-mode derivative has no truncation error."""
    import json
    import os
    with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "tangent_single_bubble.json")) as f:
        fx = json.load(f)
    p, s = single_bubble(np.float64)
    g, _ = run_adjoint(p, s, fx["steps"], 50, rain_weight(p), {})
    assert fx["J"] > 0.0
    assert np.isclose(g["objective"], fx["J"], rtol=1e-13, atol=0.0)
    errs, par = fixture_errors(fx, p, s, g)
    assert max(errs) <= FIXTURE_RTOL, errs
    for k, e in par.items():
        assert e <= FIXTURE_RTOL, (k, e)
