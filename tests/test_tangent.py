"""The forward-mode derivative of the oracle (bind.tangent, oracle/oracle_tangent.cpp) against
central differences of the oracle's Float64 step, on CPU.

The tangent instantiates the oracle's own step with dual numbers, so its J must be the Float64
oracle's J (up to the summation order of the objective), and its directional derivative must
be the limit of the central differences: at h = 1e-8 relative to each field's magnitude the
differences agree with it to about 1e-8 (truncation and rounding of the differences), on the
warm-bubble case with clouds and on shapes where the periodic wraps alias."""
import numpy as np
import pytest

from oracle import bind

from states import bubble_case, small_case
from test_adjoint import direction, oracle_J, rain_weight, shifted, state_seeds, with_constants


def central(p, s, nsteps, prec_w, seeds, v, h):
    return (oracle_J(p, shifted(s, v, h), nsteps, prec_w, seeds)
            - oracle_J(p, shifted(s, v, -h), nsteps, prec_w, seeds)) / (2 * h)


@pytest.mark.parametrize("nsteps", [1, 6])
def test_tangent_matches_central_differences(nsteps):
    p, s = bubble_case(np.float64, nx=24, nz=16)
    prec_w = rain_weight(p)
    seeds = state_seeds(p, s, 11)
    rng = np.random.default_rng(40 + nsteps)
    for _ in range(2):
        v = direction(p, s, rng)
        J, dJ = bind.tangent(p, s, nsteps, direction=v, prec_weight=prec_w, state_weight=seeds)
        assert np.isclose(J, oracle_J(p, s, nsteps, prec_w, seeds), rtol=1e-14, atol=0.0)
        fd = central(p, s, nsteps, prec_w, seeds, v, 1e-8)
        assert abs(dJ - fd) <= 1e-6 * abs(fd), (dJ, fd)
    for name, kw in (("K_auto", "d_k_auto"), ("Qc_threshold", "d_qc_threshold")):
        x0 = float(getattr(p.c, name))
        hp = 1e-4 * x0
        fd = (oracle_J(with_constants(p, **{name: x0 + hp}), s, nsteps, prec_w, seeds)
              - oracle_J(with_constants(p, **{name: x0 - hp}), s, nsteps, prec_w, seeds)) / (2 * hp)
        _, dJ = bind.tangent(p, s, nsteps, prec_weight=prec_w, state_weight=seeds, **{kw: 1.0})
        assert abs(dJ - fd) <= 1e-5 * abs(fd), (name, dJ, fd)


@pytest.mark.parametrize("nx,nz", [(2, 2), (3, 5), (5, 3)])
def test_tangent_tiny_shapes(nx, nz):
    p, s = small_case(np.float64, nx, nz, do_sf=False, do_rd=False)
    prec_w = rain_weight(p)
    seeds = state_seeds(p, s, 13)
    v = direction(p, s, np.random.default_rng(nx * 10 + nz))
    J, dJ = bind.tangent(p, s, 3, direction=v, prec_weight=prec_w, state_weight=seeds)
    assert np.isclose(J, oracle_J(p, s, 3, prec_w, seeds), rtol=1e-14, atol=0.0)
    fd = central(p, s, 3, prec_w, seeds, v, 1e-8)
    assert abs(dJ - fd) <= 1e-6 * abs(fd), (dJ, fd)


def test_tangent_is_linear_in_the_direction():
    """dJ(a v + b w) = a dJ(v) + b dJ(w) to rounding: the derivative part is a linear map."""
    p, s = bubble_case(np.float64, nx=16, nz=12)
    prec_w = rain_weight(p)
    seeds = state_seeds(p, s, 2)
    rng = np.random.default_rng(3)
    v, w = direction(p, s, rng), direction(p, s, rng)
    vw = {f: 2.0 * v[f] - 0.5 * w[f] for f in v}
    _, dv = bind.tangent(p, s, 4, direction=v, prec_weight=prec_w, state_weight=seeds)
    _, dw = bind.tangent(p, s, 4, direction=w, prec_weight=prec_w, state_weight=seeds)
    _, dvw = bind.tangent(p, s, 4, direction=vw, prec_weight=prec_w, state_weight=seeds)
    assert abs(dvw - (2.0 * dv - 0.5 * dw)) <= 1e-10 * (2.0 * abs(dv) + 0.5 * abs(dw))


def test_tangent_rejects_float32():
    p, s = bubble_case(np.float32, nx=8, nz=6)
    with pytest.raises(ValueError):
        bind.tangent(p, s, 1)


def test_golden_fixture_directions_regenerate():
    """tests/golden/tangent_single_bubble.json names its directions by seed; they must
    regenerate to the same fields (squared norms to 1e-12) for the GPU comparison to mean
    anything."""
    import json
    import os
    from moist2d_b200.adjoint_check import directions
    with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "tangent_single_bubble.json")) as f:
        fx = json.load(f)
    assert fx["steps"] == 600 and fx["J"] > 0.0 and len(fx["directions"]) == fx["dirs"]
    for (d_th, d_qv), ref in zip(directions(fx["seed"], fx["dirs"], 96, 512), fx["directions"]):
        assert np.isclose(float(np.sum(d_th * d_th)), ref["norm2_theta"], rtol=1e-12, atol=0.0)
        assert np.isclose(float(np.sum(d_qv * d_qv)), ref["norm2_qv"], rtol=1e-12, atol=0.0)


def test_tangent_with_surface_fluxes_and_radiation():
    """surface_fluxes! and gray_radiation! on (the Params defaults): the dual instantiation of
    their bulk formulas, x^4 and tanh against central differences."""
    p, s = small_case(np.float64, 12, 9, do_sf=True, do_rd=True)
    assert p.do_sf and p.do_rd
    prec_w = rain_weight(p)
    seeds = state_seeds(p, s, 17)
    v = direction(p, s, np.random.default_rng(19))
    J, dJ = bind.tangent(p, s, 3, direction=v, prec_weight=prec_w, state_weight=seeds)
    assert np.isclose(J, oracle_J(p, s, 3, prec_w, seeds), rtol=1e-14, atol=0.0)
    fd = central(p, s, 3, prec_w, seeds, v, 1e-8)
    assert dJ != 0.0
    assert abs(dJ - fd) <= 1e-6 * abs(fd), (dJ, fd)
