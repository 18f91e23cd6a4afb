"""The allocation-free column solve, through the C-ABI, against the allocating one and the oracle.

moist_implicit_correction_noalloc is for hosts that cannot let a library allocate device
memory on its own: a Julia host whose device arrays all come from CUDA.jl's memory pool, a host
that reserves a fixed device-memory budget before a run, or one that keeps other streams busy
and cannot afford cudaFree, which waits for the whole device. It works in one fixed scratch
array per GPU instead of allocating. This file checks its results bit for bit against
moist_implicit_correction (which allocates, one column per call) and against the oracle's
implicit_correction! (moist.jl:974-1030), on two calls in a row with different data, on the
smallest system (nz = 2: one unknown, no sub- or super-diagonal) and on column counts that are
not a multiple of the block size; and that calls beyond the scratch array or the level limit
are refused before any work is queued. It is named to be collected last."""
import ctypes as C

import numpy as np
import pytest

from moist2d_b200 import abi, model
from moist2d_b200._lib import lib
from moist2d_b200.params import Params
from oracle import bind

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


def _call(p, flags, ncols, bufs, dt):
    import torch
    err = C.create_string_buffer(256)
    cp = p.to_c()
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = lib().moist_implicit_correction_noalloc(C.byref(cp), p.precision, flags, ncols,
                                                 *[b.data_ptr() for b in bufs], float(dt), stream, err, 256)
    return rc, err.value


@pytest.mark.parametrize("nz,ncols", [(40, 37), (2, 300), (97, 129)])
@pytest.mark.parametrize("T,flags", MODES, ids=["f32-tri64", "f32-tri32", "f64"])
def test_noalloc_matches_allocating_entry_point_and_oracle(T, flags, nz, ncols):
    import torch
    dt = T(0.25)
    tri64 = T is np.float64 or not (flags & abi.MOIST_FLAG_TRI_NATIVE)
    for seed in (11, 12):  # two calls in a row; the second sees the first call's scratch contents
        p, (w, dw, th, r2) = _columns(T, nz, ncols, seed)
        expected = w.copy()  # the allocating entry point, one column per call
        oracle = w.copy()
        for j in range(ncols):
            col = expected[j].copy()
            model.implicit_correction(col, dw[j].copy(), th[j].copy(), r2[j].copy(), dt, p, flags=flags)
            expected[j] = col
            col = oracle[j].copy()
            bind.implicit_correction(col, dw[j].copy(), th[j].copy(), r2[j].copy(), dt, p, tri64=tri64)
            oracle[j] = col
        dev = [torch.from_numpy(a).cuda() for a in (w, dw, th, r2)]  # caller-owned device buffers
        torch.cuda.synchronize()
        rc, msg = _call(p, flags, ncols, dev, dt)
        assert rc == abi.MOIST_OK, msg
        torch.cuda.synchronize()
        got = dev[0].cpu().numpy()
        assert np.array_equal(got, expected)  # bitwise, like every other parity test here
        assert np.array_equal(got, oracle)
        assert np.array_equal(got[:, -1], w[:, -1])  # the lid face is never solved


def test_noalloc_refuses_sizes_beyond_its_limits():
    import torch
    buf = torch.zeros(16, dtype=torch.float32, device="cuda")
    before = buf.clone()
    # 2 * 127 * 5000 * 8 bytes of elimination scratch > 4 MiB
    p = Params(np.float32, Nx=2, Nz=128, H=100.0 * 128 * 1.02, dz0=100.0, z_fact=1.05)
    rc, msg = _call(p, 0, 5000, [buf] * 4, 0.1)
    assert rc == abi.MOIST_ERR_ARG and b"scratch" in msg
    # more levels than the grid vectors' room in the kernel parameters
    p = Params(np.float64, Nx=2, Nz=1100, H=10.0 * 1100 * 1.02, dz0=10.0, z_fact=1.05)
    rc, msg = _call(p, 0, 1, [buf] * 4, 0.1)
    assert rc == abi.MOIST_ERR_ARG and b"limit" in msg
    torch.cuda.synchronize()
    assert torch.equal(buf, before)  # nothing was queued
