"""Seeded test states that exercise every branch of the large step: clouds and rain present,
both signs of u and w, tiny and odd grid shapes."""
import numpy as np

from moist2d_b200.init import init_state, uniform, warm_bubble
from moist2d_b200.params import Params, State, exchange_halo


def perturb(s, p, seed, cloud=True, wind=2.0, w=0.5):
    """Add seeded cloud water, rain and velocity noise to State s (in place)."""
    T = p.T
    is0, ie0 = p.is_ - 1, p.ie
    nz, nx = p.Nz, p.Nx
    u = lambda stream: uniform(seed, stream, np.arange(nz * nx)).reshape(nx, nz).T
    rho = s.rho[:, is0:ie0].astype(np.float64)
    if cloud:
        qc = np.maximum(0.0, 2e-3 * (u(11) - 0.3))
        qr = np.maximum(0.0, 1e-3 * (u(12) - 0.5))
        qr[u(13) < 0.2] = 0.0
        s.rho_qc[:, is0:ie0] = (rho * qc).astype(T)
        s.rho_qr[:, is0:ie0] = (rho * qr).astype(T)
    s.rho_u[:, is0:ie0] += (rho * wind * (2 * u(14) - 1)).astype(T)
    ww = rho * w * (2 * u(15) - 1)
    ww[-1, :] = 0.0  # rigid lid
    s.rho_w[:, is0:ie0] = ww.astype(T)
    for f in (s.rho, s.rho_u, s.rho_w, s.rho_theta, s.rho_qv, s.rho_qc, s.rho_qr):
        exchange_halo(f, p)
    return s


def small_case(T, nx, nz, seed=7, **kw):
    """init_state! restatement on a small stretched grid, then perturbed."""
    # H slightly above nz uniform layers: the stretching then ends on the remaining-height cap
    args = dict(Nx=nx, Nz=nz, H=100.0 * nz * 1.02, dz0=100.0, z_fact=1.05, ns=3, Lx=400.0 * nx)
    args.update(kw)
    p = Params(T, **args)
    s = init_state(State(p), p, seed=seed)
    perturb(s, p, seed)
    return p, s


def bubble_case(T, seed=5, nx=64, nz=40, **kw):
    """Warm bubble on a reduced grid, perturbed so that clouds and rain are present."""
    p, s = warm_bubble(T, seed=seed, nx=nx, nz=nz)
    if kw:
        p = p.replace(**kw)
    perturb(s, p, seed)
    return p, s


INTERIOR_FIELDS = ("rho", "rho_u", "rho_w", "rho_theta", "rho_qv", "rho_qc", "rho_qr")


def compare(a, b, p, fields=INTERIOR_FIELDS + ("prec",), exact=True, rtol=0.0):
    """Max relative difference per field over the interior; asserts bitwise equality when
    exact, else the given relative tolerance (relative to the field's max magnitude)."""
    is0, ie0 = p.is_ - 1, p.ie
    report = {}
    for f in fields:
        x = getattr(a, f)
        y = getattr(b, f)
        x = x[..., is0:ie0] if x.ndim == 2 else (x[is0:ie0] if f != "theta_ref" else x)
        y = y[..., is0:ie0] if y.ndim == 2 else (y[is0:ie0] if f != "theta_ref" else y)
        scale = max(float(np.max(np.abs(y))), 1e-300)
        d = float(np.max(np.abs(x.astype(np.float64) - y.astype(np.float64)))) / scale
        report[f] = d
        if exact:
            assert np.array_equal(x, y), "%s differs: max rel %.3e" % (f, d)
        else:
            assert d <= rtol, "%s differs: max rel %.3e > %.1e" % (f, d, rtol)
    return report
