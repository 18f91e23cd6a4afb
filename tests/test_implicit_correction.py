"""implicit_correction! (moist.jl:974-1030, with solve_tridiagonal! of moist.jl:952-971) on the
device, one column per call through moist_implicit_correction, bit for bit against the
oracle's restatement: random columns on stretched grids from the smallest system (nz = 2, one
unknown) up to 128 levels, in Float32 with the FP64 and the literal Float32 elimination and in
Float64. The reference's own testset (runtests.jl:165-240) checks the residual of the rebuilt
system at a tolerance; this pins every bit."""
import numpy as np
import pytest

from moist2d_b200 import abi, model
from moist2d_b200.params import Params
from oracle import bind

pytestmark = pytest.mark.gpu

MODES = [(np.float32, 0), (np.float32, abi.MOIST_FLAG_TRI_NATIVE), (np.float64, 0)]


@pytest.mark.parametrize("nz", [2, 3, 9, 64, 128])
@pytest.mark.parametrize("T,flags", MODES, ids=["f32-tri64", "f32-tri32", "f64"])
def test_implicit_correction_bitwise_against_oracle(T, flags, nz):
    rng = np.random.default_rng(100 + nz)
    p = Params(T, Nx=2, Nz=nz, H=100.0 * nz * 1.02, dz0=100.0, z_fact=1.05)
    z = p.z.astype(np.float64)
    tri64 = T is np.float64 or not (flags & abi.MOIST_FLAG_TRI_NATIVE)
    for trial in range(8):
        theta = (300.0 + 4e-3 * z + rng.uniform(-1, 1, nz)).astype(T)
        rt2pres = (340.0 + rng.uniform(-5, 5, nz)).astype(T)
        rho_w = rng.uniform(-0.5, 0.5, nz).astype(T)
        rho_w[-1] = 0
        drho_w = rng.uniform(-1e-2, 1e-2, nz).astype(T)
        dt = T(rng.uniform(0.1, 0.5))
        a, b = rho_w.copy(), rho_w.copy()
        model.implicit_correction(a, drho_w.copy(), theta.copy(), rt2pres.copy(), dt, p, flags=flags)
        bind.implicit_correction(b, drho_w.copy(), theta.copy(), rt2pres.copy(), dt, p, tri64=tri64)
        assert np.array_equal(a, b), "trial %d: max abs %.3e" % (trial, float(np.max(np.abs(a - b))))
        assert a[-1] == rho_w[-1]  # the lid face is not part of the system
        assert not np.array_equal(a[:-1], rho_w[:-1])
