"""Per-field error of a Float32 run against the Float64 run of the same initial state.

Both runs go through the CUDA library (Float32 state with the FP64 w-p elimination, and Float64
throughout); the initial states come from the same FP64 fields, so the Float32 start is the
rounded Float64 start. Reported per field, on the interior after N large steps: the relative L2
error ||x32 - x64|| / ||x64||, the largest absolute difference and the largest |x64|, for
theta = rho_theta / rho, u and w at the cell centres (as output_history forms them,
moist.jl:1797-1810), qv, qc, qr (mixing ratios) and the accumulated surface rain prec (also
the relative error of its domain total).

A run that stops with "NaN detected in ..." before N steps (the 2048 x 128 sounding workload does
near step 900 in both precisions) is reported as such, per precision, with the step at which the
end-of-stage check fired, instead of a comparison.

    python -m moist2d_b200.precision --workload bubble --steps 1800
"""
import argparse
import json

import numpy as np

FIELDS = ("theta", "u", "w", "qv", "qc", "qr", "rain")


def diagnostics(s, p):
    """theta, u, w, qv, qc, qr on the interior (nz, nx) and prec (nx,), as float64."""
    c = slice(p.is_ - 1, p.ie)
    cm = slice(p.is_ - 2, p.ie - 1)
    f = lambda a: np.asarray(a, dtype=np.float64)
    rho = f(s.rho[:, c])
    u = (f(s.rho_u[:, c]) + f(s.rho_u[:, cm])) * 0.5 / rho
    rw = f(s.rho_w[:, c])
    w = np.empty_like(rw)
    w[1:] = (rw[1:] + rw[:-1]) * 0.5 / rho[1:]
    w[0] = rw[0] * 0.5 / rho[0]
    return {"theta": f(s.rho_theta[:, c]) / rho, "u": u, "w": w, "qv": f(s.rho_qv[:, c]) / rho,
            "qc": f(s.rho_qc[:, c]) / rho, "qr": f(s.rho_qr[:, c]) / rho, "rain": f(s.prec[c])}


def compare(d32, d64):
    out = {}
    for k in FIELDS:
        a, b = d32[k], d64[k]
        nb = float(np.linalg.norm(b))
        out[k] = {"rel_l2": float(np.linalg.norm(a - b)) / nb if nb > 0 else float(np.linalg.norm(a)),
                  "max_abs": float(np.max(np.abs(a - b))), "max_ref": float(np.max(np.abs(b)))}
    ta, tb = float(np.sum(d32["rain"])), float(np.sum(d64["rain"]))
    out["rain"]["total_rel"] = abs(ta - tb) / tb if tb > 0 else abs(ta)
    return out


def run(builder, nsteps):
    """builder(T) -> (Params, State); returns the per-field comparison after nsteps, or
    {"nan": {precision: {"step": n, "error": message}}} if a run stopped at a NaN."""
    from moist2d_b200 import model
    from moist2d_b200.params import exchange_halo
    diags, nan = {}, {}
    for T in (np.float32, np.float64):
        p, s = builder(T)
        with model.Model(p) as m:
            m.upload(s)
            done = 0
            try:
                for _ in range(nsteps):  # one large step per call: the same launches as m.step(nsteps)
                    m.step(1)
                    done += 1
            except FloatingPointError as e:
                nan[np.dtype(T).name] = {"step": done + 1, "error": str(e)}
                continue
            m.download(s)
        exchange_halo(s.rho_u, p)
        diags[T] = diagnostics(s, p)
    if nan:
        return {"nan": nan}
    return compare(diags[np.float32], diags[np.float64])


def main():
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--workload", default="bubble", choices=("bubble", "plain"))
    ap.add_argument("--steps", type=int, default=1800)
    args = ap.parse_args()
    from moist2d_b200.init import sounding_bubbles, warm_bubble
    builder = warm_bubble if args.workload == "bubble" else sounding_bubbles
    print(json.dumps({"workload": args.workload, "steps": args.steps, "fields": run(builder, args.steps)}))


if __name__ == "__main__":
    main()
