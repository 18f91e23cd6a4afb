"""GPU parity: the CUDA library against the CPU oracle through the C-ABI.

The kernels and the oracle evaluate the same expressions in the same order with the same
scalar math and no contraction, so results are compared bit for bit (all interior cells of
all prognostic fields and the accumulated rain) in Float32 (FP64 and native Thomas
elimination) and Float64."""
import numpy as np
import pytest

from moist2d_b200 import abi, model
from moist2d_b200.params import Params, State
from oracle import bind

import refsets
from impls import GpuImpl
from states import bubble_case, compare, small_case

pytestmark = pytest.mark.gpu

MODES = [(np.float32, False), (np.float32, True), (np.float64, False)]
MODE_IDS = ["f32-tri64", "f32-tri32", "f64"]


def _flags(tri_native):
    return abi.MOIST_FLAG_TRI_NATIVE if tri_native else 0


def _tri64(T, tri_native):
    return T is np.float64 or not tri_native


@pytest.mark.parametrize("testset", refsets.DEVICE_SETS, ids=[f.__name__[2:] for f in refsets.DEVICE_SETS])
@pytest.mark.parametrize("tri_native", [False, True], ids=["tri64", "tri_native"])
def test_reference_testset_gpu(testset, tri_native, FT):
    testset(GpuImpl(tri_native=tri_native), FT)


@pytest.mark.parametrize("T,tri_native", MODES, ids=MODE_IDS)
def test_microphysics_bitwise(T, tri_native):
    p, s = bubble_case(T)
    a, b = s.copy(), s.copy()
    model.cloud_microphysics(a, p)
    bind.cloud_microphysics(b, p)
    compare(a, b, p, fields=("d_rho_theta_mp", "d_rho_qv_mp", "d_rho_qc_mp", "d_rho_qr_mp"))
    assert np.any(b.d_rho_qr_mp != 0) and np.any(b.d_rho_qc_mp != 0)


@pytest.mark.parametrize("T,tri_native", MODES, ids=MODE_IDS)
def test_sedimentation_bitwise(T, tri_native):
    p, s = bubble_case(T)
    a, b = s.copy(), s.copy()
    da = model.rain_sedimentation(a, p)
    db = bind.rain_sedimentation(b, p)
    compare(a, b, p, fields=("d_rho_qr_sed",))
    is0, ie0 = p.is_ - 1, p.ie
    assert np.array_equal(da[is0:ie0], db[is0:ie0])


@pytest.mark.parametrize("T,tri_native", MODES, ids=MODE_IDS)
def test_compute_step_bitwise(T, tri_native):
    p, s0 = bubble_case(T, seed=9)
    p2, s = bubble_case(T, seed=10)  # a different current state: nonzero perturbations
    rng = np.random.default_rng(3)
    phys = [np.asfortranarray((rng.standard_normal((p.ka, p.ia)) * sc).astype(T))
            for sc in (1e-5, 1e-4, 1e-3, 1e-6, 1e-6, 1e-6)]
    a, b = s.copy(), s.copy()
    model.compute_step(phys, a, s0, p, p.dt / T(2), 4, flags=_flags(tri_native))
    bind.compute_step(phys, b, s0, p, p.dt / T(2), 4, tri64=_tri64(T, tri_native))
    compare(a, b, p, fields=("rho", "rho_u", "rho_w", "rho_theta", "rho_qv", "rho_qc", "rho_qr"))


@pytest.mark.parametrize("T,tri_native", MODES, ids=MODE_IDS)
@pytest.mark.parametrize("nsteps", [1, 5])
def test_rk3_bitwise_bubble(T, tri_native, nsteps):
    p, s = bubble_case(T)
    a, b = s.copy(), s.copy()
    model.rk3_step(a, p, nsteps, flags=_flags(tri_native))
    bind.rk3_step(b, p, nsteps, tri64=_tri64(T, tri_native))
    compare(a, b, p, fields=("rho", "rho_u", "rho_w", "rho_theta", "rho_qv", "rho_qc", "rho_qr", "prec",
                             "d_rho_qr_sed", "d_rho_theta_mp"))


@pytest.mark.parametrize("T,tri_native", MODES, ids=MODE_IDS)
@pytest.mark.parametrize("nx,nz", [(2, 2), (3, 3), (4, 4), (5, 2), (2, 5), (7, 6), (33, 9)])
def test_rk3_bitwise_small_shapes(T, tri_native, nx, nz):
    p, s = small_case(T, nx, nz, do_sf=False, do_rd=False)
    a, b = s.copy(), s.copy()
    model.rk3_step(a, p, 3, flags=_flags(tri_native))
    bind.rk3_step(b, p, 3, tri64=_tri64(T, tri_native))
    compare(a, b, p)


@pytest.mark.parametrize("T,tri_native", MODES, ids=MODE_IDS)
def test_rk3_bitwise_surface_flux_and_radiation(T, tri_native):
    """Default Params: surface fluxes and gray radiation on, 4 steps (the stale halo values the
    surface fluxes read are tracked across steps)."""
    p, s = small_case(T, 6, 8)
    assert p.do_sf and p.do_rd
    a, b = s.copy(), s.copy()
    model.rk3_step(a, p, 4, flags=_flags(tri_native))
    bind.rk3_step(b, p, 4, tri64=_tri64(T, tri_native))
    compare(a, b, p, fields=("rho", "rho_u", "rho_w", "rho_theta", "rho_qv", "rho_qc", "rho_qr", "prec",
                             "mflux", "shflux", "lhflux", "d_rho_theta_rd"))


@pytest.mark.parametrize("T", [np.float32, np.float64])
def test_nan_is_reported_like_the_reference(T):
    p, s = small_case(T, 4, 4, do_sf=False, do_rd=False)
    s.rho_qv[1, p.is_] = np.nan  # a NaN written into the uploaded state (host-side injection)
    a, b = s.copy(), s.copy()
    with pytest.raises(FloatingPointError) as eg:
        model.rk3_step(a, p, 2)
    with pytest.raises(FloatingPointError) as eo:
        bind.rk3_step(b, p, 2)
    assert str(eg.value) == str(eo.value)


def test_invalid_params_rejected():
    p = Params(np.float32, Nx=4, Nz=4, H=430.0, dz0=100.0, z_fact=1.05, halo=1)
    with pytest.raises(ValueError):
        model.rk3_step(State(p), p)
    p = Params(np.float32, Nx=1, Nz=4, H=430.0, dz0=100.0, z_fact=1.05)
    s = State(p)
    with pytest.raises(ValueError):
        model.rk3_step(s, p)


@pytest.mark.parametrize("T,tri_native", MODES, ids=MODE_IDS)
def test_tiled_tracer_sweep_matches_wavefront_and_oracle(T, tri_native):
    """Multi-tile domain (8 x 3 tiles, a partial top tile): the tiled sweep (with grid-wide passes
    and without, as dataflow), the streaming sweep, the exact wavefront and the oracle agree bit
    for bit over several steps with clouds, rain and both wind signs."""
    from moist2d_b200.init import sounding_bubbles
    from states import perturb
    p, s = sounding_bubbles(T, nx=256, nz=72, nbub=2)
    perturb(s, p, 21, wind=6.0, w=2.0)
    a, b, c, d, e = s.copy(), s.copy(), s.copy(), s.copy(), s.copy()
    model.rk3_step(a, p, 3, flags=_flags(tri_native))
    model.rk3_step(b, p, 3, flags=_flags(tri_native) | abi.MOIST_FLAG_TRACER_WAVEFRONT)
    model.rk3_step(d, p, 3, flags=_flags(tri_native) | abi.MOIST_FLAG_TRACER_STREAM)
    model.rk3_step(e, p, 3, flags=_flags(tri_native) | abi.MOIST_FLAG_TRACER_DATAFLOW)
    bind.rk3_step(c, p, 3, tri64=_tri64(T, tri_native))
    compare(a, b, p)
    compare(a, c, p)
    compare(d, c, p)
    compare(e, c, p)


@pytest.mark.parametrize("T,tri_native", MODES, ids=MODE_IDS)
@pytest.mark.parametrize("nx,nz", [(2, 2), (3, 5), (7, 33), (40, 31), (33, 64), (64, 97), (19, 256)])
def test_streaming_tracer_sweep_small_shapes(T, tri_native, nx, nz):
    """The row-streaming sweep against the oracle on shapes that put rows on both sides of warp
    boundaries, partial last warps, the largest supported height and the narrowest domain."""
    from states import perturb
    p, s = small_case(T, nx, nz)
    perturb(s, p, 5, wind=4.0, w=1.0)
    a, c = s.copy(), s.copy()
    model.rk3_step(a, p, 2, flags=_flags(tri_native) | abi.MOIST_FLAG_TRACER_STREAM)
    bind.rk3_step(c, p, 2, tri64=_tri64(T, tri_native))
    compare(a, c, p)


def test_tiled_sweep_pass_counts_are_recorded():
    import ctypes as C
    from moist2d_b200._lib import lib
    from moist2d_b200.init import sounding_bubbles
    p, s = sounding_bubbles(np.float32, nx=256, nz=64, nbub=2)
    with model.Model(p) as m:
        m.upload(s)
        m.step(2)
        counts = (C.c_int * 64)()
        assert lib().moist_tracer_pass_counts(m.ctx, counts, 64) == 0
        hist = list(counts)
    assert sum(hist) == 6  # 3 stages x 2 steps
    assert hist[0] == 0 and max(i for i, v in enumerate(hist) if v) <= 8 + 2 + 2


def test_tiled_sweep_pass_trace():
    """moist_tracer_pass_trace: one entry per sweep, positive pass durations, pass 1 recomputes
    every tile of every tracer, and the pass counts agree with moist_tracer_pass_counts."""
    import ctypes as C
    from moist2d_b200._lib import lib
    from moist2d_b200.init import sounding_bubbles
    p, s = sounding_bubbles(np.float32, nx=256, nz=64, nbub=2)
    maxrec = 32
    with model.Model(p) as m:
        m.upload(s)
        lib().moist_tracer_pass_counts(m.ctx, (C.c_int * 64)(), 64)  # reset the counters
        ns_ = (C.c_longlong * (6 * maxrec))()
        tiles = (C.c_int * (6 * maxrec))()
        npass = (C.c_int * 6)()
        assert lib().moist_tracer_pass_trace(m.ctx, 2, maxrec, ns_, tiles, npass) == 0
        counts = (C.c_int * 64)()
        assert lib().moist_tracer_pass_counts(m.ctx, counts, 64) == 0
    ntiles = (256 // 32) * (64 // 32)
    hist = [0] * 64
    for w in range(6):
        n = npass[w]
        hist[n] += 1
        assert 1 <= n <= maxrec
        assert all(ns_[w * maxrec + q] > 0 for q in range(n))
        assert tiles[w * maxrec] == 3 * ntiles
        assert all(tiles[w * maxrec + q] <= 3 * ntiles for q in range(n))
    assert hist == list(counts)


@pytest.mark.parametrize("T", [np.float32, np.float64])
@pytest.mark.parametrize("nx,nz", [(70, 40), (33, 97), (200, 33)])
def test_dataflow_tiled_sweep_partial_tiles(T, nx, nz):
    """The dataflow sweep on domains whose last tile column and row are partial, against the
    oracle."""
    from states import perturb
    p, s = small_case(T, nx, nz)
    perturb(s, p, 8, wind=5.0, w=1.5)
    a, c = s.copy(), s.copy()
    model.rk3_step(a, p, 2, flags=abi.MOIST_FLAG_TRACER_DATAFLOW)
    bind.rk3_step(c, p, 2, tri64=True)
    compare(a, c, p)
