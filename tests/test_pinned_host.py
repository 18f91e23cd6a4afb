"""Host States in page-locked memory: the library moves them by kernels that read and write the
host arrays in place (one launch for the prognostic fields) instead of staging copies. The
results must equal those of the same calls on pageable arrays bit for bit, in both directions:
upload, steps, download (with the phys tendencies, whose halo columns the caller keeps), and
moist_rk3_step_host, the reference-facing rk3_step!(s, p) on a host State."""
import ctypes as C

import numpy as np
import pytest

from moist2d_b200 import abi, model
from moist2d_b200._lib import lib
from moist2d_b200.params import STATE_FIELDS

from states import compare, small_case

pytestmark = pytest.mark.gpu


def pinned_copy(s):
    """The State s in page-locked (mapped) host arrays of the same layout."""
    import torch
    out = s.copy()
    keep = []
    for f in STATE_FIELDS:
        a = getattr(s, f)
        tdt = torch.float32 if a.dtype == np.float32 else torch.float64
        if a.ndim == 2:
            t = torch.empty((a.shape[1], a.shape[0]), dtype=tdt, pin_memory=True)
            b = t.numpy().T  # (ka, ia), column-major
        else:
            t = torch.empty(a.shape, dtype=tdt, pin_memory=True)
            b = t.numpy()
        assert t.is_pinned()
        b[...] = a
        keep.append(t)
        setattr(out, f, b)
    out._keep = keep
    return out


@pytest.mark.parametrize("T", [np.float32, np.float64], ids=["f32", "f64"])
def test_pinned_state_matches_pageable(T):
    p, s = small_case(T, 70, 33, seed=21)
    s.d_rho_theta_mp[...] = T(1e-4)  # halo columns the download must keep
    ref_in, pin_in = s.copy(), pinned_copy(s)
    with model.Model(p) as m:
        m.upload(ref_in)
        m.step(3)
        ref = m.download(s.copy())
    with model.Model(p) as m:
        m.upload(pin_in)
        m.step(3)
        got = m.download(pinned_copy(s))
    compare(got, ref, p)
    for f in STATE_FIELDS:  # whole arrays, halo columns included
        assert np.array_equal(getattr(got, f), getattr(ref, f)), f


@pytest.mark.parametrize("T", [np.float32, np.float64], ids=["f32", "f64"])
def test_pinned_rk3_step_host(T):
    p, s = small_case(T, 64, 40, seed=22)
    ref = s.copy()
    pin = pinned_copy(s)
    with model.Model(p) as m:
        for st in (ref, pin):
            h = st.to_c()
            assert lib().moist_rk3_step_host(m.ctx, C.byref(h), 2) == abi.MOIST_OK
    for f in STATE_FIELDS:
        assert np.array_equal(getattr(pin, f), getattr(ref, f)), f
    compare(ref, model.rk3_step(s.copy(), p, 2), p)
