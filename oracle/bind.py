"""ctypes binding of the CPU oracle (TEST INFRASTRUCTURE).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this module. It
wraps oracle/libmoist_oracle.so (built by oracle/Makefile), the restatement of moist.jl's
large step described in oracle/moist_oracle.hpp. Functions mutate their State arguments in
place and return None, or raise FloatingPointError("NaN detected in <field>") like the
reference's error(...) (moist.jl:1543-1577).
"""
import ctypes as C
import os
import subprocess

import numpy as np

from moist2d_b200.abi import NAN_FIELDS, moist_params, moist_state_host
from moist2d_b200.params import State

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "libmoist_oracle.so")
_lib = None


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_SO):
            build()
        L = C.CDLL(_SO)
        P, S, V, D, I = C.POINTER(moist_params), C.POINTER(moist_state_host), C.c_void_p, C.c_double, C.c_int
        L.oracle_rk3_step.argtypes = [P, I, I, S, I]
        L.oracle_history_diag.argtypes = [P, I, S, C.POINTER(V)]
        L.oracle_compute_step.argtypes = [P, I, I, C.POINTER(V), S, S, D, I]
        L.oracle_cloud_microphysics.argtypes = [P, I, S]
        L.oracle_rain_sedimentation.argtypes = [P, I, S, V]
        L.oracle_surface_fluxes.argtypes = [P, I, S]
        L.oracle_gray_radiation.argtypes = [P, I, S]
        L.oracle_implicit_correction.argtypes = [P, I, I, V, V, V, V, D]
        L.oracle_eval_helper.argtypes = [P, I, I, I, C.POINTER(D), C.POINTER(D)]
        L.oracle_limited_flux.argtypes = [P, I, I, V, V, V, I, I, C.POINTER(D)]
        L.oracle_exchange_halo.argtypes = [P, I, V]
        L.oracle_solve_tridiagonal.argtypes = [I, I, V, V, V, V]
        L.oracle_invert_T_for_thetae.argtypes = [P, I, D, D, D, C.POINTER(D)]
        L.oracle_budget_terms.argtypes = [P, I, S, V, V, V, V]
        L.oracle_tangent_run.argtypes = [P, S, C.POINTER(V), V, D, D, I, V, C.POINTER(V), C.POINTER(D),
                                         C.POINTER(D)]
        for f in ("oracle_exp_d", "oracle_log_d"):
            getattr(L, f).argtypes = [D]
            getattr(L, f).restype = D
        L.oracle_pow_d.argtypes = [D, D]
        L.oracle_pow_d.restype = D
        _lib = L
    return _lib


def _check(rc):
    if rc == -2:
        raise ValueError("oracle: invalid argument")
    if rc >= 0:
        raise FloatingPointError("NaN detected in " + NAN_FIELDS[rc])


def budget_terms(s, p):
    """Per-cell budget terms (mass, water, energy; (nz, nx) doubles) and per-column rain (nx,),
    to be summed exactly (math.fsum) for the compensated sums of moist_budget."""
    cp = p.to_c()
    h = s.to_c()
    out = [np.zeros((p.Nz, p.Nx)) for _ in range(3)] + [np.zeros(p.Nx)]
    _check(lib().oracle_budget_terms(C.byref(cp), p.precision, C.byref(h),
                                     *[o.ctypes.data_as(C.c_void_p) for o in out]))
    return out


HISTORY_FIELDS = ("u", "w", "theta", "qv", "qc", "qr", "pres", "temp", "thetae", "RH")


def history_diag(s, p):
    """output_history's primitive variables (moist.jl:1795-1835): dict of (Nz, Nx) arrays of
    type T (Fortran order, z fastest)."""
    cp = p.to_c()
    h = s.to_c()
    out = {f: np.zeros((p.Nz, p.Nx), dtype=p.T, order="F") for f in HISTORY_FIELDS}
    arr = (C.c_void_p * 10)(*[out[f].ctypes.data for f in HISTORY_FIELDS])
    _check(lib().oracle_history_diag(C.byref(cp), p.precision, C.byref(h), arr))
    return out


PROGNOSTIC = ("rho", "rho_u", "rho_w", "rho_theta", "rho_qv", "rho_qc", "rho_qr")


def tangent(p, s, nsteps, direction=None, dir_prec=None, d_k_auto=0.0, d_qc_threshold=0.0,
            prec_weight=None, state_weight=None):
    """Forward-mode derivative of nsteps Float64 large steps (oracle_tangent.cpp): returns
    (J, dJ) for J = sum(prec_weight * prec_final) + sum_f sum(state_weight[f] * S_final.f) and its
    derivative in the direction (direction[f] for the prognostic fields, dir_prec,
    d_k_auto, d_qc_threshold). s is not modified."""
    if p.T is not np.float64:
        raise ValueError("oracle.tangent: Float64 Params and State only")
    keep = []

    def arr(x, shape):
        if x is None:
            return None
        a = np.asfortranarray(np.broadcast_to(np.asarray(x, dtype=np.float64), shape))
        keep.append(a)
        return a.ctypes.data

    f2 = (p.ka, p.ia)
    direction = direction or {}
    state_weight = state_weight or {}
    dirs = (C.c_void_p * 7)(*[arr(direction.get(f), f2) for f in PROGNOSTIC])
    wts = (C.c_void_p * 7)(*[arr(state_weight.get(f), f2) for f in PROGNOSTIC])
    cp = p.to_c()
    h = s.to_c()
    J, dJ = C.c_double(), C.c_double()
    _check(lib().oracle_tangent_run(C.byref(cp), C.byref(h), dirs, arr(dir_prec, (p.ia,)), float(d_k_auto),
                                    float(d_qc_threshold), int(nsteps), arr(prec_weight, (p.ia,)), wts,
                                    C.byref(J), C.byref(dJ)))
    return J.value, dJ.value


def rk3_step(s, p, nsteps=1, tri64=False):
    """rk3_step!(s, p) applied nsteps times. tri64 selects the FP64 Thomas elimination."""
    cp = p.to_c()
    h = s.to_c()
    _check(lib().oracle_rk3_step(C.byref(cp), p.precision, int(tri64), C.byref(h), int(nsteps)))


def compute_step(phys, s, s0, p, dt, ns, tri64=False):
    """compute_step!(phys..., s, s0, p, dt, ns) with phys a sequence of six (ka, ia) arrays."""
    cp = p.to_c()
    arr = (C.c_void_p * 6)(*[np.asfortranarray(a, dtype=p.T).ctypes.data for a in phys])
    keep = [np.asfortranarray(a, dtype=p.T) for a in phys]
    arr = (C.c_void_p * 6)(*[a.ctypes.data for a in keep])
    h, h0 = s.to_c(), s0.to_c()
    _check(lib().oracle_compute_step(C.byref(cp), p.precision, int(tri64), arr, C.byref(h),
                                     C.byref(h0), float(dt), int(ns)))


def cloud_microphysics(s, p):
    cp = p.to_c()
    h = s.to_c()
    _check(lib().oracle_cloud_microphysics(C.byref(cp), p.precision, C.byref(h)))


def surface_fluxes(s, p):
    """surface_fluxes!(...) on s (moist.jl:710-752)."""
    cp = p.to_c()
    h = s.to_c()
    _check(lib().oracle_surface_fluxes(C.byref(cp), p.precision, C.byref(h)))


def gray_radiation(s, p):
    """gray_radiation!(...) on s with s.theta_ref (moist.jl:776-840)."""
    cp = p.to_c()
    h = s.to_c()
    _check(lib().oracle_gray_radiation(C.byref(cp), p.precision, C.byref(h)))


def rain_sedimentation(s, p):
    cp = p.to_c()
    h = s.to_c()
    d_prec = np.zeros(p.ia, dtype=p.T)
    _check(lib().oracle_rain_sedimentation(C.byref(cp), p.precision, C.byref(h), d_prec.ctypes.data))
    return d_prec


def implicit_correction(rho_w, drho_w, theta, rt2pres, dt, p, tri64=False):
    cp = p.to_c()
    for a in (rho_w, drho_w, theta, rt2pres):
        assert a.dtype == p.T and a.flags["C_CONTIGUOUS"]
    _check(lib().oracle_implicit_correction(C.byref(cp), p.precision, int(tri64), rho_w.ctypes.data,
                                            drho_w.ctypes.data, theta.ctypes.data,
                                            rt2pres.ctypes.data, float(dt)))


def eval_helper(p, helper, inputs, nout):
    cp = p.to_c()
    x = np.ascontiguousarray(inputs, dtype=np.float64)
    n = x.shape[0]
    out = np.zeros(n * nout, dtype=np.float64)
    _check(lib().oracle_eval_helper(C.byref(cp), p.precision, helper, n,
                                    x.ctypes.data_as(C.POINTER(C.c_double)),
                                    out.ctypes.data_as(C.POINTER(C.c_double))))
    return out.reshape(n, nout) if nout > 1 else out


def limited_flux(p, direction, scalar_rho, rho, vel, k, i):
    """compute_limited_flux_x (direction 'x') or _z ('z') at 1-based (k, i)."""
    cp = p.to_c()
    out = C.c_double()
    arrs = [np.asfortranarray(a, dtype=p.T) for a in (scalar_rho, rho, vel)]
    _check(lib().oracle_limited_flux(C.byref(cp), p.precision, 0 if direction == "x" else 1,
                                     arrs[0].ctypes.data, arrs[1].ctypes.data, arrs[2].ctypes.data,
                                     k - 1, i - 1, C.byref(out)))
    return p.T(out.value)


def exchange_halo(A, p):
    cp = p.to_c()
    assert A.flags["F_CONTIGUOUS"] and A.dtype == p.T
    _check(lib().oracle_exchange_halo(C.byref(cp), p.precision, A.ctypes.data))


def solve_tridiagonal(a, b, c, d):
    prec = 0 if a.dtype == np.float32 else 1
    _check(lib().oracle_solve_tridiagonal(prec, len(b), a.ctypes.data, b.ctypes.data, c.ctypes.data,
                                          d.ctypes.data))


def invert_T_for_thetae(qt, theta_e, p_k, p):
    cp = p.to_c()
    out = (C.c_double * 2)()
    _check(lib().oracle_invert_T_for_thetae(C.byref(cp), p.precision, float(qt), float(theta_e),
                                            float(p_k), out))
    return p.T(out[0]), p.T(out[1])


def exp_d(x):
    return lib().oracle_exp_d(float(x))


def log_d(x):
    return lib().oracle_log_d(float(x))


def pow_d(x, y):
    return lib().oracle_pow_d(float(x), float(y))


__all__ = ["State", "rk3_step", "compute_step", "cloud_microphysics", "rain_sedimentation",
           "implicit_correction", "eval_helper", "limited_flux", "exchange_halo",
           "solve_tridiagonal", "invert_T_for_thetae", "exp_d", "log_d", "pow_d", "build"]
