"""Seeded initial states.

* `philox4x32` - Philox4x32-10 counter-based generator (J. K. Salmon, M. A. Moraes, R. O. Dror,
  D. E. Shaw, "Parallel random numbers: as easy as 1, 2, 3", SC'11), vectorised in numpy.
  Replaces the reference's per-thread Xoshiro streams (moist.jl:374-375), whose output depends
  on the thread schedule.
* `init_state` - restatement of init_state! (moist.jl:351-450): reference theta profile
  (boundary layer, troposphere, stratosphere), uniform theta noise, RH profile and the
  per-column Newton iteration for discrete hydrostatic balance, with noise drawn from Philox
  keyed by (seed, i, k).
* `make_config` - the synthetic workloads the benchmarks and parity tests run: a warm moist
  bubble on a 200 x 100 grid, a 2048 x 128 analytic sounding with five warm bubbles, ensembles
  of uneven members, and the 512 x 96 single-bubble case. All inputs are synthetic and seeded.

Initial states are built in float64 numpy and rounded to the state precision at the end.
The base states satisfy the model's discrete hydrostatic balance
p_k - p_{k-1} = -g (z_k - z_{k-1}) (rho_{k-1} + rho_k) / 2 (the balance of the pressure
gradient and gravity terms of moist.jl:1271-1274), with p from the model's equation of state
p = P0 (r rho theta / P0)^(cp/cv) (moist.jl:1058). Bubbles are applied at constant pressure.
"""
import math

import numpy as np

from .params import Params, State, exchange_halo

# ---------------------------------------------------------------- Philox4x32-10

_M0, _M1 = np.uint64(0xD2511F53), np.uint64(0xCD9E8D57)
_W0, _W1 = np.uint32(0x9E3779B9), np.uint32(0xBB67AE85)
_MASK = np.uint64(0xFFFFFFFF)


def philox4x32(ctr, key, rounds=10):
    """ctr: (..., 4) uint32 counters, key: (2,) uint32 -> (..., 4) uint32 outputs."""
    c = [np.asarray(ctr[..., j], dtype=np.uint32).copy() for j in range(4)]
    k0 = np.uint32(key[0])
    k1 = np.uint32(key[1])
    with np.errstate(over="ignore"):
        for _ in range(rounds):
            p0 = _M0 * c[0].astype(np.uint64)
            p1 = _M1 * c[2].astype(np.uint64)
            hi0, lo0 = (p0 >> np.uint64(32)).astype(np.uint32), (p0 & _MASK).astype(np.uint32)
            hi1, lo1 = (p1 >> np.uint64(32)).astype(np.uint32), (p1 & _MASK).astype(np.uint32)
            c = [hi1 ^ c[1] ^ k0, lo1, hi0 ^ c[3] ^ k1, lo0]
            k0 = np.uint32(k0 + _W0)
            k1 = np.uint32(k1 + _W1)
    return np.stack(c, axis=-1)


def uniform(seed, stream, idx):
    """Uniform (0, 1) doubles for integer indices idx (any shape), keyed by (seed, stream)."""
    idx = np.asarray(idx, dtype=np.uint64)
    ctr = np.zeros(idx.shape + (4,), dtype=np.uint32)
    ctr[..., 0] = (idx & _MASK).astype(np.uint32)
    ctr[..., 1] = (idx >> np.uint64(32)).astype(np.uint32)
    ctr[..., 2] = np.uint32(stream & 0xFFFFFFFF)
    out = philox4x32(ctr, (np.uint32(seed & 0xFFFFFFFF), np.uint32(0x6D6F6973)))  # "mois"
    return (out[..., 0].astype(np.float64) + 0.5) * (1.0 / 4294967296.0)


# ---------------------------------------------------------------- thermodynamics (float64)

def _esat(Tk, c):
    Tc = Tk - float(c.T0)
    return float(c.ES0) * np.exp(float(c.A_SAT) * Tc / (float(c.B_SAT) + Tc))


def _qsat(p, Tk, c):
    es = _esat(Tk, c)
    tmp = p - (1.0 - float(c.EPSvap)) * es
    return np.where(tmp > 1e-12, float(c.EPSvap) * es / np.maximum(tmp, 1e-12), 0.0)


def _gas(qv, c):
    qd = 1.0 - qv
    r = float(c.Rd) * qd + float(c.Rv) * qv
    cp = float(c.Cpd) * qd + float(c.Cpv) * qv
    return r, cp


def _state_at_pressure(p, theta_fn, rh, c, iters=30):
    """rho, qv, theta at pressure p for theta = theta_fn(Exner) and relative humidity rh."""
    qv = np.zeros_like(p)
    for _ in range(iters):
        r, cp = _gas(qv, c)
        Pi = (p / float(c.P0)) ** (r / cp)
        th = theta_fn(Pi)
        Tk = th * Pi
        qv = np.maximum(0.0, rh * _qsat(p, Tk, c))
    r, cp = _gas(qv, c)
    Pi = (p / float(c.P0)) ** (r / cp)
    th = theta_fn(Pi)
    rho = p / (r * th * Pi)
    return rho, qv, th


def hydrostatic_columns(z, theta_fn, rh_fn, c, p_surf=1e5):
    """March up the columns: rho, qv, theta, p of shape (nz, ncol) in discrete balance.

    theta_fn(k, Pi) -> theta at level k (ncol,), rh_fn(k) -> RH at level k (ncol,)."""
    nz = len(z)
    g = float(c.GRAV)
    out_rho, out_qv, out_th, out_p = [], [], [], []
    p_prev = rho_prev = None
    for k in range(nz):
        rh = rh_fn(k)
        tfn = lambda Pi, k=k: theta_fn(k, Pi)
        if k == 0:
            dzk = float(z[0])
            p = np.full_like(rh, p_surf * math.exp(-g * dzk / (287.0 * 300.0)))
            for _ in range(60):  # p0 = p_surf - g z0 rho0
                rho, qv, th = _state_at_pressure(p, tfn, rh, c)
                p = p_surf - g * dzk * rho
        else:
            dzk = float(z[k] - z[k - 1])
            p = p_prev * math.exp(-g * dzk / (287.0 * 250.0))
            for _ in range(60):  # fixed point of p_k = p_{k-1} - g dz (rho_{k-1} + rho_k)/2
                rho, qv, th = _state_at_pressure(p, tfn, rh, c)
                p = p_prev - g * dzk * 0.5 * (rho_prev + rho)
        rho, qv, th = _state_at_pressure(p, tfn, rh, c)
        out_rho.append(rho)
        out_qv.append(qv)
        out_th.append(th)
        out_p.append(p)
        p_prev, rho_prev = p, rho
    return np.array(out_rho), np.array(out_qv), np.array(out_th), np.array(out_p)


def _fill(s, p, rho, qv, th, u):
    """Write (nz, nx) float64 interior fields into State s (T precision) and exchange halos."""
    T = p.T
    is0, ie0 = p.is_ - 1, p.ie
    s.rho[:, is0:ie0] = rho.astype(T)
    s.rho_theta[:, is0:ie0] = (rho * th).astype(T)
    s.rho_qv[:, is0:ie0] = (rho * qv).astype(T)
    s.rho_u[:, is0:ie0] = (rho * u).astype(T)
    s.rho_w[:] = 0
    s.rho_qc[:] = 0
    s.rho_qr[:] = 0
    s.prec[:] = 0
    for f in (s.rho, s.rho_u, s.rho_w, s.rho_theta, s.rho_qv, s.rho_qc, s.rho_qr):
        exchange_halo(f, p)
    return s


def _bubble_shape(x, z, xc, zc, xr, zr):
    r = np.sqrt(((x - xc) / xr) ** 2 + ((z - zc) / zr) ** 2)
    return np.where(r < 1.0, np.cos(np.pi * r * 0.5) ** 2, 0.0), r


# ---------------------------------------------------------------- init_state! restatement

def init_state(s, p, seed=1):
    """init_state!(s, p, rngs) (moist.jl:351-450) with a seeded counter-based RNG."""
    T = p.T
    z = p.z.astype(np.float64)
    nz, nx = p.Nz, p.Nx
    theta0, bl, zt = float(p.theta0), float(p.bndlayer_depth), float(p.z_tropopose)
    g1, g2 = float(p.dtheta_dz_trop), float(p.dtheta_dz_stra)
    ref = np.where(z < bl, theta0, np.where(z < zt, theta0 + g1 * (z - bl),
                                            theta0 + g1 * (zt - bl) + g2 * (z - zt)))
    s.theta_ref[:] = ref.astype(T)
    ii, kk = np.meshgrid(np.arange(nx), np.arange(nz))
    noise = float(p.theta_pert) * (uniform(seed, 0, ii * nz + kk) * 2.0 - 1.0)
    theta_init = ref[:, None] + noise
    c = p.c
    RH_surf = float(p.rel_hum_surf) / 100.0
    decay = float(p.rel_hum_decay)
    rho = np.zeros((nz, nx))
    qv = np.zeros((nz, nx))
    Rd, Rv, Cpd, Cpv, P0, g = (float(c.Rd), float(c.Rv), float(c.Cpd), float(c.Cpv),
                               float(c.P0), float(c.GRAV))
    Pi = np.ones(nx)
    p_km = None
    for k in range(nz):
        if k == 0:
            theta = (theta0 + theta_init[0]) * 0.5
            qv[k] = 0.0
            zm = 0.0
        else:
            theta = (theta_init[k - 1] + theta_init[k]) * 0.5
            qv[k] = qv[k - 1]
            zm = z[k - 1]
        qd = 1.0 - qv[k]
        r = Rd * qd + Rv * qv[k]
        cp = Cpd * qd + Cpv * qv[k]
        Pi = Pi - g * (z[k] - zm) / (cp * theta)
        p_k = P0 * Pi ** (cp / r)
        T_k = ref[k] * Pi
        rho[k] = p_k / (r * T_k)
        for _ in range(10):
            qsat = _qsat(p_k, T_k, c)
            qv_new = np.maximum(0.0, RH_surf * math.exp(-z[k] / decay) * qsat)
            qv[k] += 0.8 * (qv_new - qv[k])
            qd = 1.0 - qv[k]
            r = Rd * qd + Rv * qv[k]
            cp = Cpd * qd + Cpv * qv[k]
            cv = cp - r
            Pi = (rho[k] * r * theta_init[k] / P0) ** (r / cv)
            p_k = P0 * Pi ** (cp / r)
            T_k = ref[k] * Pi
            if k > 0:
                l = p_k - p_km + g * (z[k] - z[k - 1]) * 0.5 * (rho[k - 1] + rho[k])
                dldr = cp / cv * p_k / rho[k] + g * (z[k] - z[k - 1]) * 0.5
                rho[k] -= l / dldr
        p_km = p_k
    _fill(s, p, rho, qv, theta_init, np.full((nz, nx), float(p.u0)))
    return s


# ---------------------------------------------------------------- synthetic workloads

def _grid_params(T, nx, nz, dx, dz, ns, dt, **kw):
    return Params(T, Nx=nx, Nz=nz, Lx=nx * dx, H=nz * dz, dz0=dz, z_fact=1.0, ns=ns, dt=dt,
                  do_sf=False, do_rd=False, **kw)


def warm_bubble(T=np.float32, seed=1, nx=200, nz=100):
    """Warm moist bubble: 200 x 100 cells of 100 m, theta = 300 K neutral, surface pressure
    1000 hPa, RH 20 % outside and 95 % inside a cos^2 bubble of 2 K, radius 2 km, centred at
    x = 10 km, z = 2 km, uniform +-0.01 K seeded theta noise; dt = 1 s, ns = 6."""
    p = _grid_params(T, nx, nz, 100.0, 100.0, 6, 1.0)
    c = p.c
    z = p.z.astype(np.float64)
    x = (np.arange(nx) + 0.5) * float(p.dx)
    rho0, qv0, th0, pr = hydrostatic_columns(z, lambda k, Pi: np.full_like(Pi, 300.0),
                                             lambda k: np.full(1, 0.2), c)
    X, Z = np.meshgrid(x, z)
    shape, r = _bubble_shape(X, Z, 10e3 * nx / 200.0, 2e3, 2e3, 2e3)
    noise = 0.01 * (uniform(seed, 0, np.arange(nx * nz).reshape(nx, nz).T) * 2.0 - 1.0)
    thp = 2.0 * shape + noise
    rh = np.where(r < 1.0, 0.95, 0.2)
    P = np.repeat(pr, nx, axis=1)
    rho, qv, th = _state_at_pressure(P, lambda Pi: 300.0 + thp, rh, c)
    s = State(p)
    s.theta_ref[:] = T(300.0)
    _fill(s, p, rho, qv, th, np.zeros_like(rho))
    return p, s


def _sounding_theta(z, Pi, c):
    """theta = 300 + 43 (z/12 km)^1.25 below 12 km, isothermal (T of 12 km) above."""
    zz = np.asarray(z, dtype=np.float64)
    th = 300.0 + 43.0 * np.minimum(zz / 12e3, 1.0) ** 1.25
    return th


def sounding_columns(z, c):
    """Base state of the analytic sounding: rho, qv, theta, p of shape (nz, 1)."""
    z = np.asarray(z, dtype=np.float64)
    T12 = [None]

    def theta_fn(k, Pi):
        if z[k] <= 12e3:
            return np.full_like(Pi, 300.0 + 43.0 * (z[k] / 12e3) ** 1.25)
        return T12[0] / Pi

    def rh_fn(k):
        return np.full(1, 1.0 - 0.75 * min(z[k] / 12e3, 1.0) ** 1.25)

    # the isothermal temperature is the temperature at the top of the 12 km layer
    rho, qv, th, pr = [], [], [], []
    nz = len(z)
    klast = int(np.searchsorted(z, 12e3, side="right"))
    r0, q0, t0, p0 = hydrostatic_columns(z[:max(klast, 1)], theta_fn, rh_fn, c)
    if klast < nz:
        r, cp = _gas(q0[-1], c)
        Pi_top = (p0[-1] / float(c.P0)) ** (r / cp)
        T12[0] = float((t0[-1] * Pi_top)[0])
        r1, q1, t1, p1 = hydrostatic_columns(z, theta_fn, rh_fn, c)
        return r1, q1, t1, p1
    return r0, q0, t0, p0


def _sounding_u(z):
    return 12.0 * np.tanh(np.asarray(z, dtype=np.float64) / 3e3)


def _bubbles_state(p, base, bubbles, distinct_columns=False):
    """Apply warm bubbles [(xc, zc, r, amp)] at constant pressure to the base columns.
    distinct_columns: solve only the columns a bubble touches plus one environment column and
    copy that one to the other columns (the solve is elementwise, so the untouched columns are
    the same environment column)."""
    c = p.c
    rho0, qv0, th0, pr = base
    nx, nz = p.Nx, p.Nz
    z = p.z.astype(np.float64)
    x = (np.arange(nx) + 0.5) * float(p.dx)
    X, Z = np.meshgrid(x, z)
    thp = np.zeros((nz, nx))
    for (xc, zc, rad, amp) in bubbles:
        # periodic distance in x
        dxp = np.abs(X - xc)
        dxp = np.minimum(dxp, float(p.Lx) - dxp)
        shape, _ = _bubble_shape(dxp, Z, 0.0, zc, rad, rad)
        thp += amp * shape
    P = np.repeat(pr, nx, axis=1)
    zz = np.asarray(z, dtype=np.float64)
    rh = np.repeat(np.array([[1.0 - 0.75 * min(zk / 12e3, 1.0) ** 1.25] for zk in zz]), nx, axis=1)
    th_env = np.repeat(th0, nx, axis=1)
    # environmental theta at fixed pressure plus the perturbation
    if distinct_columns:
        touched = np.flatnonzero(np.any(thp != 0.0, axis=0))
        env = np.flatnonzero(~np.any(thp != 0.0, axis=0))
        cols = np.concatenate([touched, env[:1]])
        r_, q_, t_ = _state_at_pressure(P[:, cols], lambda Pi: th_env[:, cols] + thp[:, cols], rh[:, cols], c)
        rho, qv, th = (np.empty((nz, nx)) for _ in range(3))
        for full, part in ((rho, r_), (qv, q_), (th, t_)):
            if len(env):
                full[:, env] = part[:, -1:]
            full[:, touched] = part[:, :len(touched)]
    else:
        rho, qv, th = _state_at_pressure(P, lambda Pi: th_env + thp, rh, c)
    u = np.repeat(_sounding_u(zz)[:, None], nx, axis=1)
    s = State(p)
    s.theta_ref[:] = th0[:, 0].astype(p.T)
    _fill(s, p, rho, qv, th, u)
    return s


def sounding_bubbles(T=np.float32, seed=2, nx=2048, nz=128, dx=250.0, dz=125.0, nbub=5,
                     amp=(1.5, 2.5), rad=(1.5e3, 3e3), zc=1.5e3, ns=8, dt=2.0):
    """Analytic sounding (theta = 300 + 43 (z/12km)^1.25 K below 12 km, isothermal above;
    RH = 1 - 0.75 (z/12km)^1.25, 0.25 above; u = 12 tanh(z/3km) m/s) with a seeded row of
    warm bubbles at z = 1.5 km (amplitude and radius uniform in the given ranges)."""
    p = _grid_params(T, nx, nz, dx, dz, ns, dt)
    base = sounding_columns(p.z, p.c)
    u = uniform(seed, 1, np.arange(2 * nbub)).reshape(nbub, 2)
    Lx = float(p.Lx)
    bubbles = [((j + 0.5) * Lx / nbub, zc, rad[0] + (rad[1] - rad[0]) * u[j, 1],
                amp[0] + (amp[1] - amp[0]) * u[j, 0]) for j in range(nbub)]
    return p, _bubbles_state(p, base, bubbles)


def single_bubble(T=np.float32, seed=4, nx=512, nz=96, amp=2.0, radius=2e3, ns=8, dt=2.0):
    """512 x 96 cells of 250 m x 125 m on the analytic sounding, one 2 K bubble of 2 km radius
    at x = Lx/2, z = 1.5 km."""
    p = _grid_params(T, nx, nz, 250.0, 125.0, ns, dt)
    base = sounding_columns(p.z, p.c)
    return p, _bubbles_state(p, base, [(float(p.Lx) / 2.0, 1.5e3, radius, amp)])


_SOUNDING_CACHE = {}


def ensemble_member(T=np.float32, seed=3, member=0, nx_choices=tuple(range(256, 2049, 256)),
                    nz_choices=(64, 96, 128), ns=8, dt=2.0, amp=(1.0, 3.0), rad=(1e3, 3e3)):
    """Member m of an ensemble of uneven domains: nx, nz drawn from the choices, one bubble at
    a seeded x in (0, Lx), z = 1.5 km, amplitude and radius uniform in the given ranges."""
    u = uniform(seed, 1000 + member, np.arange(5))
    nx = int(nx_choices[min(int(u[0] * len(nx_choices)), len(nx_choices) - 1)])
    nz = int(nz_choices[min(int(u[1] * len(nz_choices)), len(nz_choices) - 1)])
    p = _grid_params(T, nx, nz, 250.0, 125.0, ns, dt)
    key = (np.dtype(T).str, p.z.tobytes())
    if key not in _SOUNDING_CACHE:  # the hydrostatic march depends on the grid only
        _SOUNDING_CACHE[key] = sounding_columns(p.z, p.c)
    base = _SOUNDING_CACHE[key]
    bub = [(u[2] * float(p.Lx), 1.5e3, rad[0] + (rad[1] - rad[0]) * u[4],
            amp[0] + (amp[1] - amp[0]) * u[3])]
    return p, _bubbles_state(p, base, bub, distinct_columns=True)


# ---------------------------------------------------------------- the library's generators
#
# The same workloads built by the C-ABI generators (moist_init_*, include/moist2d.h), which a
# caller of the shared library without Python (a Julia host) uses. They agree with the numpy
# versions above to the last bits of double-precision exp / pow before the final rounding.

def _lib():
    from ._lib import lib
    return lib()


def _check(rc, what):
    if rc != 0:
        raise ValueError("%s failed with status %d" % (what, rc))


def uniform_lib(seed, stream, idx):
    """uniform(seed, stream, idx) through moist_uniform."""
    import ctypes as C
    idx = np.ascontiguousarray(np.asarray(idx, dtype=np.uint64).ravel())
    out = np.zeros(idx.size)
    _check(_lib().moist_uniform(int(seed), int(stream), idx.size, idx.ctypes.data_as(C.POINTER(C.c_uint64)),
                                out.ctypes.data_as(C.POINTER(C.c_double))), "moist_uniform")
    return out


def warm_bubble_lib(T=np.float32, seed=1, nx=200, nz=100):
    """warm_bubble through moist_init_warm_bubble."""
    p = _grid_params(T, nx, nz, 100.0, 100.0, 6, 1.0)
    s = State(p)
    cp = p.to_c()
    h = s.to_c()
    import ctypes as C
    _check(_lib().moist_init_warm_bubble(C.byref(cp), p.precision, int(seed), C.byref(h)), "moist_init_warm_bubble")
    return p, s


def _bubbles_lib(p, bubbles):
    import ctypes as C
    from .abi import moist_bubble
    arr = (moist_bubble * max(1, len(bubbles)))()
    for j, (xc, zc, rad, amp) in enumerate(bubbles):
        arr[j].xc, arr[j].zc, arr[j].radius, arr[j].amp = xc, zc, rad, amp
    s = State(p)
    cp = p.to_c()
    h = s.to_c()
    _check(_lib().moist_init_sounding(C.byref(cp), p.precision, arr, len(bubbles), C.byref(h)),
           "moist_init_sounding")
    return s


def sounding_bubbles_lib(T=np.float32, seed=2, nx=2048, nz=128, dx=250.0, dz=125.0, nbub=5,
                         amp=(1.5, 2.5), rad=(1.5e3, 3e3), zc=1.5e3, ns=8, dt=2.0):
    """sounding_bubbles through moist_sounding_bubble_row and moist_init_sounding."""
    import ctypes as C
    from .abi import moist_bubble
    p = _grid_params(T, nx, nz, dx, dz, ns, dt)
    row = (moist_bubble * nbub)()
    _check(_lib().moist_sounding_bubble_row(int(seed), nbub, float(p.Lx), amp[0], amp[1], rad[0], rad[1], zc, row),
           "moist_sounding_bubble_row")
    return p, _bubbles_lib(p, [(b.xc, b.zc, b.radius, b.amp) for b in row])


def ensemble_member_lib(T=np.float32, seed=3, member=0, nx_choices=tuple(range(256, 2049, 256)),
                        nz_choices=(64, 96, 128), ns=8, dt=2.0, amp=(1.0, 3.0), rad=(1e3, 3e3)):
    """ensemble_member through moist_ensemble_member_draw and moist_init_sounding."""
    import ctypes as C
    from .abi import moist_bubble
    nxc = (C.c_int * len(nx_choices))(*nx_choices)
    nzc = (C.c_int * len(nz_choices))(*nz_choices)
    nx, nz, b = C.c_int(), C.c_int(), moist_bubble()
    _check(_lib().moist_ensemble_member_draw(int(seed), int(member), nxc, len(nx_choices), nzc, len(nz_choices),
                                             250.0, amp[0], amp[1], rad[0], rad[1], 1.5e3, C.byref(nx),
                                             C.byref(nz), C.byref(b)), "moist_ensemble_member_draw")
    p = _grid_params(T, nx.value, nz.value, 250.0, 125.0, ns, dt)
    return p, _bubbles_lib(p, [(b.xc, b.zc, b.radius, b.amp)])


def init_state_lib(s, p, seed=1):
    """init_state through moist_init_state (the fields of p that init_state! reads)."""
    import ctypes as C
    from .abi import moist_init_profile
    prof = moist_init_profile()
    for f, g in (("theta0", "theta0"), ("bndlayer_depth", "bndlayer_depth"), ("z_tropopause", "z_tropopose"),
                 ("dtheta_dz_trop", "dtheta_dz_trop"), ("dtheta_dz_stra", "dtheta_dz_stra"),
                 ("theta_pert", "theta_pert"), ("rel_hum_surf", "rel_hum_surf"),
                 ("rel_hum_decay", "rel_hum_decay"), ("u0", "u0")):
        setattr(prof, f, float(getattr(p, g)))
    cp = p.to_c()
    h = s.to_c()
    _check(_lib().moist_init_state(C.byref(cp), p.precision, C.byref(prof), int(seed), C.byref(h)), "moist_init_state")
    return s
