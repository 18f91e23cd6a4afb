"""The shared scalar math (moist2d_b200/csrc/moist_math.h) against glibc: exp <= 1 ulp,
log <= 1 ulp, pow <= 2 ulp over the argument ranges the model uses and beyond."""
import math

import numpy as np

from oracle import bind


def _ulps(got, ref):
    return abs(got - ref) / math.ulp(ref) if ref != 0 else abs(got)


def test_exp_within_one_ulp():
    rng = np.random.default_rng(1)
    xs = np.concatenate([rng.uniform(-30, 30, 20000), rng.uniform(-700, 700, 5000), [0.0, 1.0, -1.0]])
    assert max(_ulps(bind.exp_d(x), math.exp(x)) for x in xs) <= 1.0


def test_log_within_one_ulp():
    rng = np.random.default_rng(2)
    xs = np.concatenate([10 ** rng.uniform(-300, 300, 10000), rng.uniform(0.5, 2.0, 10000), [1.0, 2.0]])
    assert max(_ulps(bind.log_d(x), math.log(x)) for x in xs) <= 1.0


def test_pow_within_two_ulp():
    rng = np.random.default_rng(3)
    x = 10 ** rng.uniform(-12, 3, 20000)   # covers (rho_qr/rho)^0.1346 and the Exner powers
    y = rng.uniform(-5, 5, 20000)
    assert max(_ulps(bind.pow_d(a, b), a ** b) for a, b in zip(x, y)) <= 2.0
    assert bind.pow_d(2.0, 0.0) == 1.0 and bind.pow_d(0.0, 2.0) == 0.0 and math.isnan(bind.pow_d(-1.0, 0.5))


def test_model_arguments():
    # Exner function and pressure at typical states: (r rho theta / P0)^(r/cv), Pi^(cp/r)
    for base, e in ((0.86, 0.4), (0.99, 3.5), (1.2e-4, 0.1346)):
        assert _ulps(bind.pow_d(base, e), base ** e) <= 1.0
