"""Gradient check of moist_adjoint_run on the adjoint workload.

Workload: 512 x 96 cells of 250 m x 125 m on the analytic sounding, one 2 K bubble of 2 km
radius at x = Lx/2, z = 1.5 km, dt = 2 s, ns = 8; objective J = total surface rain
sum(prec * dx) after N large steps; checkpoints every C steps. The Float64 gradient with respect
to the initial theta' field (rho_theta at fixed rho), the initial qv (rho_qv at fixed rho),
K_auto and Qc_threshold is compared with central differences of the library's Float64 step
(bitwise equal to the oracle's) on seeded random directions; the Float32 gradient (Float32
trajectory, double adjoint) is compared with the Float64 one.

Directions are random combinations of four large-scale modes sin(2 pi kx x / Lx + phase)
sin(pi kz (k + 1/2) / nz), kx in 1..5, kz in 1..3, seeded, scaled to O(1 K) in theta' and
O(1e-4) in qv. Over hundreds of steps of moist convection the objective is only piecewise
smooth (limiter, upwind and saturation switches in every cell), and along cell-by-cell white
noise the central differences themselves do not converge as h shrinks (they scatter by about
10 % between h = 1e-4 and 1e-9 over 600 steps), so white-noise directions (--white) check the
differences more than the adjoint.

    python -m moist2d_b200.adjoint_check --steps 600 --ckpt 50 --dirs 64
"""
import argparse
import json
import time

import numpy as np

from . import model
from .init import single_bubble
from .params import Constants


def rain_weight(p):
    w = np.zeros(p.ia)
    w[p.is_ - 1:p.ie] = float(p.dx)
    return w


def run(p, s, nsteps, ckpt):
    with model.Model(p) as m:
        m.upload(s)
        return m.adjoint(nsteps, ckpt, prec_weight=rain_weight(p))


def objective(p, s, nsteps):
    with model.Model(p) as m:
        m.upload(s)
        m.step(nsteps)
        out = s.copy()
        m.download(out)
    return float(np.sum(rain_weight(p) * out.prec.astype(np.float64)))


def controls(p, s, g):
    """Gradients w.r.t. theta' (theta at fixed rho: d/dtheta = rho d/drho_theta) and qv (at
    fixed rho: rho d/drho_qv), interior only."""
    c = slice(p.is_ - 1, p.ie)
    rho = s.rho[:, c].astype(np.float64)
    return {"theta": rho * g["rho_theta"][:, c], "qv": rho * g["rho_qv"][:, c]}


def directions(seed, n, nz, nx, white=False):
    """n seeded (d_theta, d_qv) pairs of (nz, nx) fields: each a random combination of four
    large-scale modes sin(2 pi kx x / Lx + phase) sin(pi kz (k + 1/2) / nz) (kx in 1..5, kz in
    1..3), or white noise; d_qv scaled by 1e-4. Drawn in the order d_theta, d_qv, d_theta, ..."""
    rng = np.random.default_rng(seed)
    zz, xx = np.meshgrid(np.arange(nz), np.arange(nx), indexing="ij")

    def field():
        if white:
            return rng.standard_normal((nz, nx))
        d = np.zeros((nz, nx))
        for _ in range(4):
            kx, kz, ph = rng.integers(1, 6), rng.integers(1, 4), rng.uniform(0.0, 2.0 * np.pi)
            d += rng.standard_normal() * np.sin(2 * np.pi * kx * xx / nx + ph) * np.sin(np.pi * kz * (zz + 0.5) / nz)
        return d

    out = []
    for _ in range(n):
        d_th = field()
        out.append((d_th, 1e-4 * field()))
    return out


def state_direction(p, s, d_theta, d_qv):
    """The State-space direction of (d_theta, d_qv) at fixed rho: d rho_theta = rho d_theta,
    d rho_qv = rho d_qv on the interior, as (ka, ia) arrays with zero halo columns."""
    c = slice(p.is_ - 1, p.ie)
    rho = s.rho[:, c].astype(np.float64)
    out = {}
    for f, d in (("rho_theta", d_theta), ("rho_qv", d_qv)):
        a = np.zeros((p.ka, p.ia))
        a[:, c] = rho * d
        out[f] = a
    return out


def perturbed(p, s, d_theta, d_qv, h):
    a = s.copy()
    c = slice(p.is_ - 1, p.ie)
    rho = s.rho[:, c].astype(np.float64)
    a.rho_theta[:, c] = (s.rho_theta[:, c].astype(np.float64) + h * rho * d_theta).astype(s.rho_theta.dtype)
    a.rho_qv[:, c] = (s.rho_qv[:, c].astype(np.float64) + h * rho * d_qv).astype(s.rho_qv.dtype)
    return a


def main():
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--steps", type=int, default=600)
    ap.add_argument("--ckpt", type=int, default=50)
    ap.add_argument("--dirs", type=int, default=64)
    ap.add_argument("--h", type=float, default=1e-7, help="relative step of the central differences")
    ap.add_argument("--seed", type=int, default=3)
    ap.add_argument("--white", action="store_true", help="white-noise directions instead of large-scale modes")
    args = ap.parse_args()

    p64, s64 = single_bubble(np.float64)
    p32, s32 = single_bubble(np.float32)
    t0 = time.perf_counter()
    g64 = run(p64, s64, args.steps, args.ckpt)
    t1 = time.perf_counter()
    g32 = run(p32, s32, args.steps, args.ckpt)
    cg64, cg32 = controls(p64, s64, g64), controls(p32, s32, g32)

    errs = []
    for d_th, d_qv in directions(args.seed, args.dirs, p64.Nz, p64.Nx, args.white):
        ad = float(np.sum(cg64["theta"] * d_th) + np.sum(cg64["qv"] * d_qv))
        h = args.h
        fd = (objective(p64, perturbed(p64, s64, d_th, d_qv, h), args.steps)
              - objective(p64, perturbed(p64, s64, d_th, d_qv, -h), args.steps)) / (2 * h)
        errs.append({"adjoint": ad, "fd": fd, "rel": abs(ad - fd) / max(abs(fd), 1e-300)})
    par = {}
    for name, key in (("K_auto", "k_auto"), ("Qc_threshold", "qc_threshold")):
        x0 = float(getattr(p64.c, name))
        hp = 1e-4 * x0

        def with_c(x):
            kw = {k: float(getattr(p64.c, k)) for k in ("K_auto", "Qc_threshold")}
            kw[name] = x
            return p64.replace(constants=Constants(np.float64, **kw))

        fd = (objective(with_c(x0 + hp), s64, args.steps) - objective(with_c(x0 - hp), s64, args.steps)) / (2 * hp)
        par[name] = {"adjoint": g64[key], "fd": fd, "rel": abs(g64[key] - fd) / max(abs(fd), 1e-300),
                     "f32_adjoint": g32[key], "f32_rel": abs(g32[key] - g64[key]) / max(abs(g64[key]), 1e-300)}
    rel = np.array([e["rel"] for e in errs]) if errs else np.zeros(1)
    f32 = {k: float(np.linalg.norm(cg32[k] - cg64[k]) / max(np.linalg.norm(cg64[k]), 1e-300)) for k in cg64}
    print(json.dumps({
        "workload": "single bubble 512x96, dt=2 s, ns=8, rain objective", "steps": args.steps,
        "ckpt_every": args.ckpt, "objective_f64": g64["objective"], "objective_f32": g32["objective"],
        "f64_ms": {"forward": g64["forward_ms"], "reverse": g64["reverse_ms"]},
        "f32_ms": {"forward": g32["forward_ms"], "reverse": g32["reverse_ms"],
                   "ratio": g32["reverse_ms"] / g32["forward_ms"]},
        "fd": {"directions": args.dirs, "kind": "white noise" if args.white else "large-scale modes", "h": args.h, "max_rel": float(np.max(rel)),
               "median_rel": float(np.median(rel)), "frac_le_1e-3": float(np.mean(rel <= 1e-3)),
               "worst": sorted(errs, key=lambda e: -e["rel"])[:3]},
        "params": par, "f32_vs_f64_rel_l2": f32, "wall_s": time.perf_counter() - t0,
        "adjoint_f64_wall_s": t1 - t0}))


if __name__ == "__main__":
    main()
