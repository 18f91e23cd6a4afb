"""The allocation-free column solve against the allocating one, through the C-ABI.

moist_implicit_correction_noalloc exists for callers that cannot let a library allocate
device memory: a Julia host whose device arrays all come from CUDA.jl's memory pool, or code
that runs while its stream is being captured into a CUDA graph, where cudaMalloc is not
allowed. It works in one fixed scratch array per GPU instead of allocating. This file checks
its results against moist_implicit_correction (which allocates) on two calls in a row with
different data, and that oversized calls are refused before any work is queued. It is named
to be collected last."""
import ctypes as C

import numpy as np
import pytest

from moist2d_b200 import abi, model
from moist2d_b200._lib import lib
from moist2d_b200.params import Params

pytestmark = pytest.mark.gpu

MODES = [(np.float32, 0), (np.float32, abi.MOIST_FLAG_TRI_NATIVE), (np.float64, 0)]


def _columns(T, nz, ncols, seed):
    rng = np.random.default_rng(seed)
    p = Params(T, Nx=2, Nz=nz, H=100.0 * nz * 1.02, dz0=100.0, z_fact=1.05)
    z = p.z.astype(np.float64)
    theta = 300.0 + 4e-3 * z[None, :] + rng.uniform(-1, 1, (ncols, nz))
    rt2pres = 340.0 + rng.uniform(-5, 5, (ncols, nz))
    rho_w = rng.uniform(-0.5, 0.5, (ncols, nz))
    rho_w[:, -1] = 0.0
    drho_w = rng.uniform(-1e-2, 1e-2, (ncols, nz))
    # (ncols, nz) C order = (nz, ncols) with z fastest, the reference layout
    return p, [np.ascontiguousarray(a.astype(T)) for a in (rho_w, drho_w, theta, rt2pres)]


@pytest.mark.parametrize("T,flags", MODES, ids=["f32-tri64", "f32-tri32", "f64"])
def test_noalloc_matches_allocating_entry_point(T, flags):
    import torch
    nz, ncols = 40, 37
    dt = T(0.25)
    for seed in (11, 12):  # two calls in a row; the second sees the first call's scratch contents
        p, (w, dw, th, r2) = _columns(T, nz, ncols, seed)
        expected = w.copy()
        for j in range(ncols):
            col = expected[j].copy()
            model.implicit_correction(col, dw[j].copy(), th[j].copy(), r2[j].copy(), dt, p, flags=flags)
            expected[j] = col
        dev = [torch.from_numpy(a).cuda() for a in (w, dw, th, r2)]  # caller-owned device buffers
        torch.cuda.synchronize()
        cp = p.to_c()
        err = C.create_string_buffer(256)
        stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
        rc = lib().moist_implicit_correction_noalloc(C.byref(cp), p.precision, flags, ncols,
                                                     dev[0].data_ptr(), dev[1].data_ptr(),
                                                     dev[2].data_ptr(), dev[3].data_ptr(),
                                                     float(dt), stream, err, 256)
        assert rc == abi.MOIST_OK, err.value
        torch.cuda.synchronize()
        got = dev[0].cpu().numpy()
        assert np.array_equal(got, expected)  # bitwise, like every other parity test here


def test_noalloc_refuses_sizes_beyond_its_scratch():
    import torch
    nz, ncols = 128, 5000  # 2 * 127 * 5000 * 8 bytes > 4 MiB
    p = Params(np.float32, Nx=2, Nz=nz, H=100.0 * nz * 1.02, dz0=100.0, z_fact=1.05)
    buf = torch.zeros(16, dtype=torch.float32, device="cuda")
    cp = p.to_c()
    err = C.create_string_buffer(256)
    rc = lib().moist_implicit_correction_noalloc(C.byref(cp), p.precision, 0, ncols, buf.data_ptr(),
                                                 buf.data_ptr(), buf.data_ptr(), buf.data_ptr(), 0.1,
                                                 None, err, 256)
    assert rc == abi.MOIST_ERR_ARG
    assert b"scratch" in err.value
