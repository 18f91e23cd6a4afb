"""The reference's testsets (runtests.jl) run against the CPU oracle: this pins the oracle."""
import pytest

import refsets
from impls import OracleImpl

ALL = refsets.DEVICE_SETS + refsets.HOST_ONLY_SETS


@pytest.mark.parametrize("testset", ALL, ids=[f.__name__[2:] for f in ALL])
@pytest.mark.parametrize("tri64", [False, True], ids=["tri_native", "tri_fp64"])
def test_reference_testset_oracle(testset, tri64, FT):
    testset(OracleImpl(tri64=tri64), FT)
