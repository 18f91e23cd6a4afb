import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built library")
    config.addinivalue_line("markers", "slow: long-running CPU test")


@pytest.fixture(scope="session", autouse=True)
def _build_oracle():
    from oracle import bind
    bind.build()
    yield


@pytest.fixture(params=[np.float32, np.float64], ids=["Float32", "Float64"])
def FT(request):
    """The precision argument of `julia test/runtests.jl [Float32|Float64]`."""
    return request.param


def tol(FT, f32, f64=None):
    """tol(f32, f64=f32*1e-6) of runtests.jl:23."""
    if f64 is None:
        f64 = f32 * 1e-6
    return FT(f64) if FT is np.float64 else FT(f32)


def isapprox(x, y, FT, atol=0.0, rtol=None):
    """Julia isapprox: |x - y| <= max(atol, rtol * max(|x|, |y|)) (norms for arrays); rtol
    defaults to sqrt(eps(T)) unless atol > 0."""
    if rtol is None:
        rtol = 0.0 if atol > 0 else float(np.sqrt(np.finfo(FT).eps))
    x = np.asarray(x, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    if x.ndim == 0:
        return bool(x == y or abs(x - y) <= max(atol, rtol * max(abs(x), abs(y))))
    return bool(np.linalg.norm(x - y) <= max(atol, rtol * max(np.linalg.norm(x), np.linalg.norm(y))))
