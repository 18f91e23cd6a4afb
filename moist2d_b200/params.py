"""Host-side mirror of the reference's configuration and state types.

`Params` restates `Params{T}` and its constructor (moist.jl:70-222) and the physical
constants of `set_constants!` (moist.jl:26-60), evaluated in the state precision T exactly as
Julia does (every default and derived value is rounded to T and combined in T arithmetic).
`State` restates `State` / `allocate_state` (moist.jl:294-345): (ka, ia) column-major
(Fortran-order) numpy arrays, z fastest.

One deliberate extension: `Params(..., dt=...)` takes the large time step explicitly. The
reference's constructor always recomputes dt from CFL = 0.6 and `tout_int`
(moist.jl:184-195); callers there use `Parameters.reconstruct(p; dt=...)` or the field
constructor `Params{T}(; dt=...)`, which is what `dt=` stands for here.
"""
import ctypes as C
import math

import numpy as np

from .abi import STATE_FIELDS, moist_params, moist_state_host, MOIST_F32, MOIST_F64


def precision_of(T):
    T = np.dtype(T).type
    if T is np.float32:
        return MOIST_F32
    if T is np.float64:
        return MOIST_F64
    raise ValueError("precision must be float32 or float64")


class Constants:
    """set_constants!(T) (moist.jl:26-60): every value rounded to T, derived values in T."""

    def __init__(self, T=np.float32, **override):
        T = np.dtype(T).type
        self.T = T
        v = dict(GRAV=9.81, Rd=287.04, Rv=461.5, Cpd=1004.64, Cpv=1846.0, Cpl=4218.0,
                 P0=1e5, Lv=2.501e6, Ka=0.4, SIGMA=5.67e-8,
                 K_auto=1e-3, Qc_threshold=1e-3, K_accr=2.2, K_evap=1e-2, A_term=36.3,
                 B_term=0.1346, T0=273.15, ES0=610.78, A_SAT=17.67, B_SAT=243.5, EPS=1e-12)
        v.update(override)
        for k, x in v.items():
            setattr(self, k, T(x))
        self.Cvd = T(self.Cpd - self.Rd)
        self.EPSvap = T(self.Rd / self.Rv)
        self.EPSTvap = T(self.Rv / self.Rd - T(1.0))


class Params:
    """Params{T} (moist.jl:70-178) built like `Params(T; kwargs...)` (moist.jl:180-222)."""

    _defaults = dict(
        Lx=160e3, H=25e3, Nx=640, Nz=250, halo=2, dz0=50.0, z_fact=1.02, nu=1.0, Pr=0.7,
        gamma_d=0.1, beta_offcenter=1.0, zf_sponge=0.2,
        do_mp=True, do_auto=True, do_accr=True, do_revap=True, do_sed=True, do_rd=True,
        do_sf=True,
        Cd=1.2e-3, Ch=0.8e-3, Ce=1.0e-3, uabs_min=5.0, temp_surf=300.0, k_abs_qv=0.15,
        k_abs_qc=20.0, k_abs_qr=10.0, surf_emissivity=1.0, tau_cooling=864000.0, u0=0.0,
        theta0=300.0, bndlayer_depth=1000.0, z_tropopose=15e3, dtheta_dz_trop=4.0e-3,
        dtheta_dz_stra=18.3e-3, theta_pert=2.0, rel_hum_surf=90.0, rel_hum_decay=4000.0,
        t_end=86400.0 * 2.0, tout_int=300.0, ns=3,
    )
    _real = ("Lx", "H", "dz0", "z_fact", "nu", "Pr", "gamma_d", "beta_offcenter", "zf_sponge",
             "Cd", "Ch", "Ce", "uabs_min", "temp_surf", "k_abs_qv", "k_abs_qc", "k_abs_qr",
             "surf_emissivity", "tau_cooling", "u0", "theta0", "bndlayer_depth", "z_tropopose",
             "dtheta_dz_trop", "dtheta_dz_stra", "theta_pert", "rel_hum_surf", "rel_hum_decay")

    def __init__(self, T=np.float32, constants=None, dt=None, dx=None, kappa=None, check_grid=True,
                 **kw):
        T = np.dtype(T).type
        self.T = T
        unknown = set(kw) - set(self._defaults)
        if unknown:
            raise TypeError("unknown Params fields: %s" % sorted(unknown))
        v = dict(self._defaults)
        v.update(kw)
        for k in self._real:
            v[k] = T(v[k])
        for k in ("Nx", "Nz", "halo", "ns"):
            v[k] = int(v[k])
        self.__dict__.update(v)
        self.c = constants if constants is not None else Constants(T)
        self.ia = self.Nx + 2 * self.halo
        self.ka = self.Nz
        self.is_ = 1 + self.halo          # 1-based, as in the reference
        self.ie = self.Nx + self.halo
        self.ks = 1
        self.ke = self.Nz
        self.dx = T(dx) if dx is not None else T(self.Lx / T(self.Nx))
        self.kappa = T(kappa) if kappa is not None else T(self.nu / self.Pr)
        # time step (moist.jl:183-195), unless given explicitly
        CFL, cs = 0.6, 340.0
        dt_raw = CFL * float(self.dx) * self.ns / cs
        self.Nint_steps = math.ceil(self.tout_int / dt_raw)
        self.dt = T(dt) if dt is not None else T(self.tout_int / self.Nint_steps)
        self.N_steps = math.ceil(self.t_end / float(self.dt))
        # axes (moist.jl:198-216), in T arithmetic
        ia, ka = self.ia, self.ka
        half = T(0.5)
        self.x = np.array([T(T(i - self.is_) + half) * self.dx for i in range(1, ia + 1)], dtype=T)
        zf = np.zeros(ka, dtype=T)
        dz = np.zeros(ka, dtype=T)
        z = np.zeros(ka, dtype=T)
        zf[0] = self.dz0
        dz[0] = self.dz0
        z[0] = T(zf[0] * half)
        for k in range(1, ka):            # 0-based k = reference k - 1
            kk = k + 1
            a = T(dz[k - 1] * self.z_fact)
            b = T(T(self.H - zf[k - 1]) / T(self.ke - kk + 1))
            dz[k] = a if a <= b else b
            zf[k] = T(zf[k - 1] + dz[k])
            z[k] = T(T(zf[k - 1] + zf[k]) * half)
        # check_grid=False mirrors the field constructor Params{T}(; ...), which skips the grid
        if check_grid and zf[ka - 1] < self.H:
            raise ValueError("z_fact is too small: %r, %r < %r" % (self.z_fact, zf[ka - 1], self.H))
        self.zf, self.dz, self.z = zf, dz, z
        self._c = None

    @property
    def precision(self):
        return precision_of(self.T)

    def replace(self, **kw):
        """Parameters.reconstruct(p; kw...) equivalent."""
        base = {k: getattr(self, k) for k in self._defaults}
        base.update(dt=self.dt, constants=self.c)
        base.update(kw)
        return Params(self.T, **base)

    def to_c(self):
        """moist_params for the C-ABI (grid vectors referenced, not copied: keep self alive)."""
        c = self.c
        p = moist_params()
        p.nx, p.nz, p.halo, p.ns = self.Nx, self.Nz, self.halo, self.ns
        p.lx, p.h, p.dx = float(self.Lx), float(self.H), float(self.dx)
        p.zf = self.zf.ctypes.data
        p.dz = self.dz.ctypes.data
        p.z = self.z.ctypes.data
        p.dt = float(self.dt)
        p.nu, p.kappa, p.gamma_d = float(self.nu), float(self.kappa), float(self.gamma_d)
        p.beta_offcenter, p.zf_sponge = float(self.beta_offcenter), float(self.zf_sponge)
        for f in ("do_mp", "do_auto", "do_accr", "do_revap", "do_sed", "do_rd", "do_sf"):
            setattr(p, f, int(bool(getattr(self, f))))
        p.cd, p.ch, p.ce = float(self.Cd), float(self.Ch), float(self.Ce)
        p.uabs_min, p.temp_surf = float(self.uabs_min), float(self.temp_surf)
        p.k_abs_qv, p.k_abs_qc, p.k_abs_qr = float(self.k_abs_qv), float(self.k_abs_qc), float(self.k_abs_qr)
        p.surf_emissivity, p.tau_cooling = float(self.surf_emissivity), float(self.tau_cooling)
        p.z_tropopause = float(self.z_tropopose)
        p.grav, p.rd, p.rv, p.cpd = float(c.GRAV), float(c.Rd), float(c.Rv), float(c.Cpd)
        p.cpv, p.cpl, p.cvd, p.p0 = float(c.Cpv), float(c.Cpl), float(c.Cvd), float(c.P0)
        p.lv, p.sigma, p.epsvap = float(c.Lv), float(c.SIGMA), float(c.EPSvap)
        p.k_auto, p.qc_threshold, p.k_accr = float(c.K_auto), float(c.Qc_threshold), float(c.K_accr)
        p.k_evap, p.a_term, p.b_term = float(c.K_evap), float(c.A_term), float(c.B_term)
        p.t0, p.es0, p.a_sat, p.b_sat, p.eps = float(c.T0), float(c.ES0), float(c.A_SAT), float(c.B_SAT), float(c.EPS)
        self._c = p
        return p


_2D = ("rho", "rho_u", "rho_w", "rho_theta", "rho_qv", "rho_qc", "rho_qr",
       "d_rho_theta_mp", "d_rho_qv_mp", "d_rho_qc_mp", "d_rho_qr_mp", "d_rho_qr_sed",
       "d_rho_theta_rd")
_1DX = ("prec", "mflux", "shflux", "lhflux", "d_rho_u_sf", "d_rho_theta_sf", "d_rho_qv_sf")


class State:
    """State / allocate_state (moist.jl:294-345): zero-filled (ka, ia) Fortran-order arrays."""

    def __init__(self, p):
        T = p.T
        for f in _2D:
            setattr(self, f, np.zeros((p.ka, p.ia), dtype=T, order="F"))
        for f in _1DX:
            setattr(self, f, np.zeros(p.ia, dtype=T))
        self.theta_ref = np.zeros(p.ka, dtype=T)

    def copy(self):
        s = State.__new__(State)
        for f in STATE_FIELDS:
            setattr(s, f, getattr(self, f).copy(order="K"))
        return s

    def to_c(self, fields=STATE_FIELDS):
        h = moist_state_host()
        for f in fields:
            a = getattr(self, f)
            assert a.flags["F_CONTIGUOUS"] or a.ndim == 1
            setattr(h, f, a.ctypes.data)
        return h


def exchange_halo(A, p):
    """exchange_halo!(A, p) (moist.jl:233-241) on a (ka, ia) numpy array."""
    h, ie, is_ = p.halo, p.ie, p.is_
    if h == 0:
        return A
    left = A[:, ie - h:ie].copy()
    right = A[:, is_ - 1:is_ - 1 + h].copy()
    A[:, 0:h] = left
    A[:, ie:ie + h] = right
    return A
