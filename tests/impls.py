"""Implementation adapters for the restated reference testsets (tests/refsets.py).

`OracleImpl` runs the CPU oracle; `GpuImpl` runs the CUDA library through its C-ABI. Both
expose the reference-shaped calls the testsets need; State arguments are mutated in place.
"""
import numpy as np

from oracle import bind


class OracleImpl:
    name = "oracle"

    def __init__(self, tri64=False):
        self.tri64 = tri64

    def eval_helper(self, p, helper, inputs, nout):
        return bind.eval_helper(p, helper, inputs, nout)

    def implicit_correction(self, rho_w, drho_w, theta, rt2pres, dt, p):
        bind.implicit_correction(rho_w, drho_w, theta, rt2pres, dt, p, tri64=self.tri64)

    def compute_step(self, phys, s, s0, p, dt, ns):
        bind.compute_step(phys, s, s0, p, dt, ns, tri64=self.tri64)

    def rk3_step(self, s, p, nsteps=1):
        bind.rk3_step(s, p, nsteps, tri64=self.tri64)

    def cloud_microphysics(self, s, p):
        bind.cloud_microphysics(s, p)

    def exchange_halo(self, A, p):
        bind.exchange_halo(A, p)

    def solve_tridiagonal(self, a, b, c, d):
        bind.solve_tridiagonal(a, b, c, d)

    def limited_flux(self, p, direction, scalar_rho, rho, vel, k, i):
        return bind.limited_flux(p, direction, scalar_rho, rho, vel, k, i)

    def invert_T_for_thetae(self, qt, theta_e, p_k, p):
        return bind.invert_T_for_thetae(qt, theta_e, p_k, p)


class GpuImpl:
    name = "gpu"

    def __init__(self, tri_native=False):
        self.tri_native = tri_native

    def _flags(self):
        from moist2d_b200 import abi
        return abi.MOIST_FLAG_TRI_NATIVE if self.tri_native else 0

    def eval_helper(self, p, helper, inputs, nout):
        from moist2d_b200 import model
        return model.eval_helper(p, helper, inputs, nout)

    def implicit_correction(self, rho_w, drho_w, theta, rt2pres, dt, p):
        from moist2d_b200 import model
        model.implicit_correction(rho_w, drho_w, theta, rt2pres, dt, p, flags=self._flags())

    def compute_step(self, phys, s, s0, p, dt, ns):
        from moist2d_b200 import model
        model.compute_step(phys, s, s0, p, dt, ns, flags=self._flags())

    def rk3_step(self, s, p, nsteps=1):
        from moist2d_b200 import model
        model.rk3_step(s, p, nsteps, flags=self._flags())

    def cloud_microphysics(self, s, p):
        from moist2d_b200 import model
        model.cloud_microphysics(s, p)
