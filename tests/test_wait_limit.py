"""Bounded device-side waits: a wait that runs out ends the step with MOIST_ERR_TIMEOUT instead of
hanging, and the context stays usable.

The tiled tracer sweep's blocks wait for each other between repair passes, or, in its dataflow
form, for their left and lower neighbours' new strips (the reference's in-place sweep,
moist.jl:1469-1518, has no such wait; its threads never synchronise). Here the
wait limit is set to one SM clock cycle, so that waits give up almost at once; nothing faults
and nothing spins without bound. The same context, with the default limit restored and the
State uploaded again, then steps bit for bit like the oracle."""
import ctypes as C

import numpy as np
import pytest

from moist2d_b200 import abi, model
from moist2d_b200._lib import lib
from moist2d_b200.init import sounding_bubbles
from oracle import bind

from states import compare

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("flags", [0, abi.MOIST_FLAG_TRACER_DATAFLOW], ids=["passes", "dataflow"])
def test_wait_that_runs_out_returns_timeout_and_context_recovers(flags):
    p, s = sounding_bubbles(np.float32, nx=512, nz=96, nbub=2)
    with model.Model(p, flags=flags) as m:
        assert lib().moist_set_wait_limit(m.ctx, 1) == abi.MOIST_OK
        m.upload(s)
        rc = lib().moist_rk3_step(m.ctx, 2)
        assert rc == abi.MOIST_ERR_TIMEOUT
        assert b"timed out" in lib().moist_last_error(m.ctx)
        # default limit again, a fresh State: the context steps like the oracle
        assert lib().moist_set_wait_limit(m.ctx, 0) == abi.MOIST_OK
        m.upload(s)
        m.step(2)
        a = m.download(s.copy())
    b = s.copy()
    bind.rk3_step(b, p, 2, tri64=True)
    compare(a, b, p)
    # a fresh context is unaffected
    c = s.copy()
    model.rk3_step(c, p, 2, flags=flags)
    compare(c, b, p)


def test_wait_limit_unsupported_without_waiting_kernels():
    p, s = sounding_bubbles(np.float32, nx=64, nz=32, nbub=1)
    with model.Model(p, flags=abi.MOIST_FLAG_TRACER_STREAM) as m:
        assert lib().moist_set_wait_limit(m.ctx, 1) == abi.MOIST_ERR_UNSUPPORTED
