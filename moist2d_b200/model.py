"""Reference-shaped host API over the CUDA library.

The functions mirror moist.jl's entry points (same names, argument meaning and in-place
semantics): `rk3_step(s, p)` (moist.jl:1589), `compute_step(phys, s, s0, p, dt, ns)` (1039),
`cloud_microphysics(s, p)` (554), `rain_sedimentation(s, p)` (674),
`implicit_correction(rho_w, drho_w, theta, rt2pres, dt, p)` (974). A NaN found by the
end-of-stage check raises FloatingPointError("NaN detected in <field>"), the counterpart of the
reference's error(...) (moist.jl:1543-1577).

`Model` keeps a State resident on the device between calls (the reference's device() hook,
moist.jl:227-228): upload once, step many times, download when needed.
"""
import ctypes as C

import numpy as np

from . import abi
from ._lib import lib


def _raise(rc, ctx=None, what=""):
    if rc == abi.MOIST_OK:
        return
    L = lib()
    msg = L.moist_last_error(ctx).decode() if ctx else L.moist_status_string(rc).decode()
    if rc == abi.MOIST_ERR_NAN:
        raise FloatingPointError(msg)
    if rc == abi.MOIST_ERR_ARG:
        raise ValueError("%s: invalid argument %s" % (what, msg))
    if rc == abi.MOIST_ERR_UNSUPPORTED:
        raise NotImplementedError("%s: %s" % (what, msg))
    if rc == abi.MOIST_ERR_IO:
        raise OSError("%s: %s" % (what, L.moist_io_last_error().decode()))
    raise RuntimeError("%s failed (%s): %s" % (what, L.moist_status_string(rc).decode(), msg))


class Model:
    """A device-resident State with its Params (one CUDA stream)."""

    def __init__(self, p, flags=0):
        self.p = p
        self._cp = p.to_c()
        self.flags = flags
        self.ctx = C.c_void_p()
        _raise(lib().moist_ctx_create(C.byref(self._cp), p.precision, flags, C.byref(self.ctx)),
               None, "moist_ctx_create")

    def close(self):
        if self.ctx:
            lib().moist_ctx_destroy(self.ctx)
            self.ctx = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def upload(self, s):
        h = s.to_c()
        _raise(lib().moist_upload_state(self.ctx, C.byref(h)), self.ctx, "moist_upload_state")

    def download(self, s):
        h = s.to_c()
        _raise(lib().moist_download_state(self.ctx, C.byref(h)), self.ctx, "moist_download_state")
        return s

    def step(self, nsteps=1):
        _raise(lib().moist_rk3_step(self.ctx, int(nsteps)), self.ctx, "moist_rk3_step")

    def time_steps(self, nsteps):
        ms = C.c_float()
        _raise(lib().moist_time_steps(self.ctx, int(nsteps), C.byref(ms)), self.ctx, "moist_time_steps")
        return ms.value

    def budget(self):
        out = (C.c_double * 4)()
        _raise(lib().moist_budget(self.ctx, out), self.ctx, "moist_budget")
        return np.array(out[:])

    def synchronize(self):
        _raise(lib().moist_synchronize(self.ctx), self.ctx, "moist_synchronize")

    @property
    def nan_field(self):
        return lib().moist_nan_field(self.ctx)

    HISTORY_FIELDS = ("u", "w", "theta", "qv", "qc", "qr", "pres", "temp", "thetae", "RH")

    def history(self, fields=HISTORY_FIELDS):
        """output_history's primitive variables from the device State (moist_history_diagnostics):
        dict of the requested fields as (Nz, Nx) arrays (z fastest) plus "summary": min w,
        max w, max qc (g/kg), max qr (g/kg), min RH, max RH."""
        p = self.p
        out = {f: np.zeros((p.Nz, p.Nx), dtype=p.T, order="F") for f in fields}
        arr = (C.c_void_p * abi.MOIST_NDIAG)(*[out[f].ctypes.data if f in out else None
                                               for f in self.HISTORY_FIELDS])
        summ = (C.c_double * 6)()
        _raise(lib().moist_history_diagnostics(self.ctx, arr, summ), self.ctx, "moist_history_diagnostics")
        out["summary"] = dict(zip(("w_min", "w_max", "qc_max_gkg", "qr_max_gkg", "rh_min", "rh_max"), summ[:]))
        return out

    def autotune(self, nsteps=3):
        """moist_autotune: time every strip width and exact tracer sweep from the current State,
        keep the fastest, restore the State; returns the report (timings and choice)."""
        buf = C.create_string_buffer(2048)
        _raise(lib().moist_autotune(self.ctx, int(nsteps), buf, len(buf)), self.ctx, "moist_autotune")
        return buf.value.decode()

    def set_adjoint_tapes(self, mode):
        """moist_set_adjoint_tapes: 1 a tape per step of a checkpoint segment, 0 one tape and
        the segment's States, -1 (default) chosen from the free device memory."""
        _raise(lib().moist_set_adjoint_tapes(self.ctx, int(mode)), self.ctx, "moist_set_adjoint_tapes")

    def adjoint(self, nsteps, ckpt_every=50, prec_weight=None, state_seed=None):
        """Advance the resident State nsteps large steps and return the gradient of
        J = sum(prec_weight * prec_final) + sum_f sum(state_seed[f] * S_final.f)
        (moist_adjoint_run). prec_weight: (ia,) array or None; state_seed: dict from the
        prognostic field names (rho, rho_u, rho_w, rho_theta, rho_qv, rho_qc, rho_qr) to (ka, ia)
        arrays. Returns a dict: the gradients w.r.t. the initial fields as (ka, ia) float64 arrays
        (halo columns 0), "prec", "k_auto", "qc_threshold", "objective", "forward_ms",
        "reverse_ms". The Model is left at the final State."""
        p = self.p
        ka, ia = p.ka, p.ia
        keep = []

        def f64(a, shape):
            a = np.asfortranarray(np.asarray(a, dtype=np.float64))
            if a.shape != shape:
                raise ValueError("seed of shape %s, expected %s" % (a.shape, shape))
            keep.append(a)
            return a.ctypes.data

        seed = abi.moist_adjoint_seed()
        if prec_weight is not None:
            seed.prec_weight = f64(prec_weight, (ia,))
        for j, name in enumerate(abi.PROGNOSTIC):
            if state_seed is not None and name in state_seed:
                seed.state[j] = f64(state_seed[name], (ka, ia))
        grads = {name: np.zeros((ka, ia), dtype=np.float64, order="F") for name in abi.PROGNOSTIC}
        grads["prec"] = np.zeros(ia, dtype=np.float64)
        out = abi.moist_adjoint_grad()
        for j, name in enumerate(abi.PROGNOSTIC):
            out.state[j] = grads[name].ctypes.data
        out.prec = grads["prec"].ctypes.data
        _raise(lib().moist_adjoint_run(self.ctx, int(nsteps), int(ckpt_every), C.byref(seed), C.byref(out)),
               self.ctx, "moist_adjoint_run")
        grads.update(k_auto=out.k_auto, qc_threshold=out.qc_threshold, objective=out.objective,
                     forward_ms=out.forward_ms, reverse_ms=out.reverse_ms)
        return grads


def rk3_step(s, p, nsteps=1, flags=0):
    """rk3_step!(s, p) applied nsteps times; s is updated in place."""
    with Model(p, flags) as m:
        m.upload(s)
        try:
            m.step(nsteps)
        finally:
            m.download(s)
    return s


def compute_step(phys, s, s0, p, dt, ns, flags=0):
    """compute_step!(phys..., s, s0, p, dt, ns); phys = six (ka, ia) arrays in the reference order."""
    keep = [np.asfortranarray(a, dtype=p.T) for a in phys]
    arr = (C.c_void_p * 6)(*[a.ctypes.data for a in keep])
    h0 = s0.to_c()
    with Model(p, flags) as m:
        m.upload(s)
        try:
            _raise(lib().moist_compute_step(m.ctx, arr, C.byref(h0), float(dt), int(ns)), m.ctx,
                   "moist_compute_step")
        finally:
            m.download(s)
    return s


def cloud_microphysics(s, p):
    """cloud_microphysics!(d_rho_qv_mp, ..., rho, ..., p): fills s.d_rho_*_mp."""
    with Model(p) as m:
        m.upload(s)
        _raise(lib().moist_cloud_microphysics(m.ctx), m.ctx, "moist_cloud_microphysics")
        m.download(s)
    return s


def surface_fluxes(s, p):
    """surface_fluxes!(d_rho_u_sf, d_rho_theta_sf, d_rho_qv_sf, mflux, shflux, lhflux, rho, ...,
    p): fills those six fields of s (the halo columns of s are the reads at is-1 and ie+1)."""
    with Model(p) as m:
        m.upload(s)
        _raise(lib().moist_surface_fluxes(m.ctx), m.ctx, "moist_surface_fluxes")
        m.download(s)
    return s


def gray_radiation(s, p):
    """gray_radiation!(d_rho_theta_rd, rho, ..., theta_ref, p): fills s.d_rho_theta_rd."""
    with Model(p) as m:
        m.upload(s)
        _raise(lib().moist_gray_radiation(m.ctx), m.ctx, "moist_gray_radiation")
        m.download(s)
    return s


def rain_sedimentation(s, p):
    """rain_sedimentation!(d_rho_qr_sed, d_prec, rho_qr, rho, p): fills s.d_rho_qr_sed and
    returns d_prec."""
    d_prec = np.zeros(p.ia, dtype=p.T)
    with Model(p) as m:
        m.upload(s)
        _raise(lib().moist_rain_sedimentation(m.ctx, d_prec.ctypes.data), m.ctx,
               "moist_rain_sedimentation")
        m.download(s)
    return d_prec


def implicit_correction(rho_w, drho_w, theta, rt2pres, dt, p, flags=0):
    cp = p.to_c()
    for a in (rho_w, drho_w, theta, rt2pres):
        assert a.dtype == p.T and a.flags["C_CONTIGUOUS"]
    _raise(lib().moist_implicit_correction(C.byref(cp), p.precision, flags, rho_w.ctypes.data,
                                           drho_w.ctypes.data, theta.ctypes.data,
                                           rt2pres.ctypes.data, float(dt)), None,
           "moist_implicit_correction")


def eval_helper(p, helper, inputs, nout):
    cp = p.to_c()
    x = np.ascontiguousarray(inputs, dtype=np.float64)
    n = x.shape[0]
    out = np.zeros(n * nout, dtype=np.float64)
    _raise(lib().moist_eval_helper(C.byref(cp), p.precision, helper, n,
                                   x.ctypes.data_as(C.POINTER(C.c_double)),
                                   out.ctypes.data_as(C.POINTER(C.c_double))), None,
           "moist_eval_helper")
    return out.reshape(n, nout) if nout > 1 else out


class Ensemble:
    """Independent domains advanced together (moist_batch_*): one launch per kernel of the large
    step for all members, each step a CUDA graph. `params` are the members' Params (one
    precision; ns, do_sf and do_rd equal; nz <= 256). Every member's results equal those of a
    Model stepping that member alone, bit for bit."""

    def __init__(self, params, flags=0):
        self.params = list(params)
        precs = {p.precision for p in self.params}
        if len(precs) != 1:
            raise ValueError("Ensemble: members of one precision")
        self._cps = [p.to_c() for p in self.params]
        arr = (abi.moist_params * len(self._cps))(*self._cps)
        self.b = C.c_void_p()
        rc = lib().moist_batch_create(arr, len(self._cps), precs.pop(), flags, C.byref(self.b))
        _raise(rc, None, "moist_batch_create")

    def close(self):
        if self.b:
            lib().moist_batch_destroy(self.b)
            self.b = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, rc, what):
        if rc == abi.MOIST_OK:
            return
        msg = lib().moist_batch_last_error(self.b).decode()
        if rc == abi.MOIST_ERR_NAN:
            raise FloatingPointError(msg)
        raise RuntimeError("%s failed (%s): %s" % (what, lib().moist_status_string(rc).decode(), msg))

    def member(self, i):
        return lib().moist_batch_member(self.b, int(i))

    def upload(self, i, s):
        h = s.to_c()
        ctx = self.member(i)
        _raise(lib().moist_batch_upload(self.b, int(i), C.byref(h)), ctx, "moist_batch_upload")

    def download(self, i, s):
        h = s.to_c()
        ctx = self.member(i)
        _raise(lib().moist_batch_download(self.b, int(i), C.byref(h)), ctx, "moist_batch_download")
        return s

    def step(self, nsteps=1):
        self._check(lib().moist_batch_step(self.b, int(nsteps)), "moist_batch_step")

    def time_steps(self, nsteps):
        ms = C.c_float()
        self._check(lib().moist_batch_time_steps(self.b, int(nsteps), C.byref(ms)), "moist_batch_time_steps")
        return ms.value

    def profile(self, nsteps):
        """(total ms, per-group ms) of nsteps launched without the graphs (MOIST_KGROUP_* order)."""
        tot = C.c_float()
        g = (C.c_float * abi.MOIST_NGROUPS)()
        self._check(lib().moist_batch_profile(self.b, int(nsteps), C.byref(tot), g), "moist_batch_profile")
        return tot.value, list(g)

    @property
    def nan_member(self):
        return lib().moist_batch_nan_member(self.b)

    def autotune(self, nsteps=2):
        """moist_batch_autotune: time the per-column kernels' block sizes from the current
        States, keep the fastest, restore the States; returns the report."""
        buf = C.create_string_buffer(1024)
        self._check(lib().moist_batch_autotune(self.b, int(nsteps), buf, len(buf)), "moist_batch_autotune")
        return buf.value.decode()

    def adjoint(self, nsteps, ckpt_every=50, prec_weights=None, state_seeds=None, nthreads=0):
        """moist_batch_adjoint_run: Model.adjoint for every member. nthreads = 0: the members'
        kernels run packed (one launch per kernel for all members); nthreads > 0: every member's
        own moist_adjoint_run from that many host threads. prec_weights / state_seeds: per-member
        lists (entries as for Model.adjoint) or None. Returns one gradient dict per member;
        every member is left at its final State."""
        n = len(self.params)
        keep = []

        def f64(a, shape):
            a = np.asfortranarray(np.asarray(a, dtype=np.float64))
            if a.shape != shape:
                raise ValueError("seed of shape %s, expected %s" % (a.shape, shape))
            keep.append(a)
            return a.ctypes.data

        seeds = (abi.moist_adjoint_seed * n)()
        outs = (abi.moist_adjoint_grad * n)()
        grads = []
        for m, p in enumerate(self.params):
            ka, ia = p.ka, p.ia
            if prec_weights is not None and prec_weights[m] is not None:
                seeds[m].prec_weight = f64(prec_weights[m], (ia,))
            sd = state_seeds[m] if state_seeds is not None else None
            g = {name: np.zeros((ka, ia), dtype=np.float64, order="F") for name in abi.PROGNOSTIC}
            g["prec"] = np.zeros(ia, dtype=np.float64)
            for j, name in enumerate(abi.PROGNOSTIC):
                if sd is not None and name in sd:
                    seeds[m].state[j] = f64(sd[name], (ka, ia))
                outs[m].state[j] = g[name].ctypes.data
            outs[m].prec = g["prec"].ctypes.data
            grads.append(g)
        self._check(lib().moist_batch_adjoint_run(self.b, int(nsteps), int(ckpt_every), seeds, outs, int(nthreads)),
                    "moist_batch_adjoint_run")
        for m, g in enumerate(grads):
            o = outs[m]
            g.update(k_auto=o.k_auto, qc_threshold=o.qc_threshold, objective=o.objective,
                     forward_ms=o.forward_ms, reverse_ms=o.reverse_ms)
        return grads

    def set_adjoint_tapes(self, mode):
        """moist_batch_set_adjoint_tapes (modes as for Model.set_adjoint_tapes)."""
        self._check(lib().moist_batch_set_adjoint_tapes(self.b, int(mode)), "moist_batch_set_adjoint_tapes")

    def budget(self, i):
        out = (C.c_double * 4)()
        ctx = self.member(i)
        _raise(lib().moist_budget(ctx, out), ctx, "moist_budget")
        return np.array(out[:])


class History:
    """init_history / output_history (moist.jl:1716-1891): a NetCDF history file (classic format
    with 64-bit offsets, written by the library) with the reference's dimensions, variables,
    units and element type. `append(t, model)` writes one record from a Model's device State
    (diagnostics computed on the device); `append_host(t, s, diag)` writes it from a host State
    and the ten diagnostics as Model.history returns them."""

    FIELDS = Model.HISTORY_FIELDS

    def __init__(self, path, p):
        self.p = p
        self._cp = p.to_c()
        self.h = C.c_void_p()
        _raise(lib().moist_history_create(str(path).encode(), C.byref(self._cp), p.precision, C.byref(self.h)),
               None, "moist_history_create")

    def append(self, t, model):
        _raise(lib().moist_history_append(self.h, float(t), model.ctx), model.ctx, "moist_history_append")

    def append_member(self, t, ensemble, i):
        """One record from member i of an Ensemble (its member context, after Ensemble.step)."""
        ctx = ensemble.member(i)
        _raise(lib().moist_history_append(self.h, float(t), ctx), ctx, "moist_history_append")

    def append_host(self, t, s, diag):
        p = self.p
        keep = []

        def arr(f):
            a = np.asfortranarray(np.asarray(diag[f], dtype=p.T))
            if a.shape != (p.Nz, p.Nx):
                raise ValueError("diagnostic %s of shape %s, expected %s" % (f, a.shape, (p.Nz, p.Nx)))
            keep.append(a)
            return a.ctypes.data

        d = (C.c_void_p * abi.MOIST_NDIAG)(*[arr(f) for f in self.FIELDS])
        h = s.to_c()
        _raise(lib().moist_history_append_host(self.h, float(t), C.byref(h), d), None, "moist_history_append_host")

    def close(self):
        if self.h:
            rc = lib().moist_history_close(self.h)
            self.h = C.c_void_p()
            _raise(rc, None, "moist_history_close")

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def restart_read(path, p, s=None):
    """The restart of run_sim (moist.jl:1905-1919): the State of the last record of a history
    file (rho, rho_u, rho_w, rho_theta = theta * rho, rho_qv, rho_qc, rho_qr = q * rho, prec;
    periodic halo columns), into s or a new zero State. rho_qr comes from "qr" (the reference
    reads "qc" there, moist.jl:1917)."""
    from .params import State
    if s is None:
        s = State(p)
    cp = p.to_c()
    h = s.to_c()
    _raise(lib().moist_restart_read(str(path).encode(), C.byref(cp), p.precision, C.byref(h)), None,
           "moist_restart_read")
    return s
