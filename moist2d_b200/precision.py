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

--control replaces the Float32 run by a second Float64 run whose initial rho_theta differs from
the first in the last bit (every cell one ulp up or down, seeded): the spread two Float64 runs
reach from a last-bit difference is the floor below which no Float32 error can be read as a
precision effect once the flow amplifies rounding differences.

--workload ensemble runs the 256 uneven members of the batched workload (nx in {256, ..., 2048},
nz in {64, 96, 128}, one seeded bubble each on the analytic sounding) through moist_batch_* in
both precisions and reports, per member, the relative error of its domain-total accumulated rain
and the relative L2 error of its per-column rain; a member that stops at a NaN in either
precision is listed with the step instead.

    python -m moist2d_b200.precision --workload bubble --steps 1800 [--control]
    python -m moist2d_b200.precision --workload ensemble --steps 1800
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


def last_bit_perturbed(s, p, seed=17):
    """s with every interior rho_theta moved one ulp up or down (seeded), in place."""
    from .init import uniform
    c = slice(p.is_ - 1, p.ie)
    a = s.rho_theta[:, c]
    up = uniform(seed, 7, np.arange(a.size)).reshape(a.shape) < 0.5
    s.rho_theta[:, c] = np.where(up, np.nextafter(a, np.inf), np.nextafter(a, -np.inf))
    return s


def run(builder, nsteps, control=False):
    """builder(T) -> (Params, State); returns the per-field comparison after nsteps, or
    {"nan": {precision: {"step": n, "error": message}}} if a run stopped at a NaN. control: the
    first run is Float64 from a last-bit-perturbed start instead of Float32."""
    from moist2d_b200 import model
    from moist2d_b200.params import exchange_halo
    diags, nan = {}, {}
    runs = (("float64-perturbed", np.float64), ("float64", np.float64)) if control else \
        (("float32", np.float32), ("float64", np.float64))
    for name, T in runs:
        p, s = builder(T)
        if name == "float64-perturbed":
            last_bit_perturbed(s, p)
        with model.Model(p) as m:
            m.upload(s)
            done = 0
            try:
                for _ in range(nsteps):  # one large step per call: the same launches as m.step(nsteps)
                    m.step(1)
                    done += 1
            except FloatingPointError as e:
                nan[name] = {"step": done + 1, "error": str(e)}
                continue
            m.download(s)
        exchange_halo(s.rho_u, p)
        diags[name] = diagnostics(s, p)
    if nan:
        return {"nan": nan}
    return compare(diags[runs[0][0]], diags["float64"])


def run_ensemble(nmem, nsteps, seed=3):
    """Per-member rain of the batched workload in Float32 against Float64 after nsteps."""
    from moist2d_b200 import model
    from moist2d_b200.init import ensemble_member
    rain, nan = {}, {}
    for T in (np.float32, np.float64):
        name = np.dtype(T).name
        mem = [ensemble_member(T, seed=seed, member=m) for m in range(nmem)]
        stopped = {}
        with model.Ensemble([p for p, _ in mem]) as e:
            for i, (_, s) in enumerate(mem):
                e.upload(i, s)
            for n in range(nsteps):
                try:
                    e.step(1)
                except FloatingPointError as err:
                    m = e.nan_member
                    if m not in stopped:
                        stopped[m] = {"step": n + 1, "error": str(err)}
                    # a stopped member stays stopped; the others keep stepping
            rain[name] = []
            for i, (p, s) in enumerate(mem):
                e.download(i, s)
                rain[name].append(np.asarray(s.prec[p.is_ - 1:p.ie], dtype=np.float64))
        nan[name] = stopped
    members = []
    for i in range(nmem):
        if i in nan["float32"] or i in nan["float64"]:
            members.append({"member": i, "nan": {k: v[i] for k, v in nan.items() if i in v}})
            continue
        a, b = rain["float32"][i], rain["float64"][i]
        ta, tb = float(np.sum(a)), float(np.sum(b))
        nb = float(np.linalg.norm(b))
        members.append({"member": i, "nx": int(a.size), "rain_total_f64": tb,
                        "total_rel": abs(ta - tb) / tb if tb > 0 else abs(ta),
                        "column_rel_l2": float(np.linalg.norm(a - b)) / nb if nb > 0 else float(np.linalg.norm(a))})
    ok = [m for m in members if "nan" not in m and m["rain_total_f64"] > 0]
    tot = np.array([m["total_rel"] for m in ok]) if ok else np.zeros(0)
    summary = {"members": nmem, "compared": len(ok), "nan_members": sum("nan" in m for m in members),
               "total_rel_median": float(np.median(tot)) if tot.size else None,
               "total_rel_max": float(np.max(tot)) if tot.size else None,
               "total_rel_le_1e-4": int(np.sum(tot <= 1e-4))}
    return {"summary": summary, "members": members}


def main():
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--workload", default="bubble", choices=("bubble", "plain", "ensemble"))
    ap.add_argument("--steps", type=int, default=1800)
    ap.add_argument("--members", type=int, default=256)
    ap.add_argument("--control", action="store_true",
                    help="Float64 from a last-bit-perturbed start against Float64, instead of Float32")
    args = ap.parse_args()
    from moist2d_b200.init import sounding_bubbles, warm_bubble
    if args.workload == "ensemble":
        print(json.dumps({"workload": "ensemble", "steps": args.steps,
                          "rain": run_ensemble(args.members, args.steps)}))
        return
    builder = warm_bubble if args.workload == "bubble" else sounding_bubbles
    print(json.dumps({"workload": args.workload, "steps": args.steps, "control": args.control,
                      "fields": run(builder, args.steps, control=args.control)}))


if __name__ == "__main__":
    main()
