"""Generates tests/golden/tangent_single_bubble.json: exact directional derivatives of the adjoint
workload's objective, computed by the forward-mode (dual-number) oracle (oracle/oracle_tangent.cpp).

Workload: moist2d_b200.init.single_bubble(Float64) (512 x 96, one 2 K bubble, dt = 2 s, ns = 8),
J = total surface rain sum(prec * dx) after STEPS large steps. Directions: the seeded
large-scale (d_theta, d_qv) pairs of moist2d_b200.adjoint_check.directions at fixed rho, plus
the two Kessler parameters K_auto and Qc_threshold. The fixture holds, per direction, dJ/dv and
the squared norms of the two fields (so a test can tell that it regenerated the same
directions), and J itself. tests/test_adjoint.py compares the library's Float64 adjoint with it.

    python tests/golden/make_tangent_single_bubble.py --steps 600 --dirs 16 --procs 8

Each direction is one Float64 forward run with one dual derivative (about 3 minutes on one core
at 600 steps); the runs go to a pool of worker processes.
"""
import argparse
import json
import multiprocessing as mp
import os
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tangent_single_bubble.json")


def _task(args):
    kind, index, seed, ndirs, steps = args
    from moist2d_b200.adjoint_check import directions, rain_weight, state_direction
    from moist2d_b200.init import single_bubble
    from oracle import bind
    p, s = single_bubble(np.float64)
    w = rain_weight(p)
    if kind == "dir":
        d_th, d_qv = directions(seed, ndirs, p.Nz, p.Nx)[index]
        J, dJ = bind.tangent(p, s, steps, direction=state_direction(p, s, d_th, d_qv), prec_weight=w)
        return kind, index, J, dJ, float(np.sum(d_th * d_th)), float(np.sum(d_qv * d_qv))
    kw = {"k_auto": "d_k_auto", "qc_threshold": "d_qc_threshold"}[index]
    J, dJ = bind.tangent(p, s, steps, prec_weight=w, **{kw: 1.0})
    return kind, index, J, dJ, None, None


def main():
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--steps", type=int, default=600)
    ap.add_argument("--dirs", type=int, default=16)
    ap.add_argument("--seed", type=int, default=3)
    ap.add_argument("--procs", type=int, default=os.cpu_count() or 1)
    args = ap.parse_args()
    tasks = [("dir", j, args.seed, args.dirs, args.steps) for j in range(args.dirs)]
    tasks += [("param", k, args.seed, args.dirs, args.steps) for k in ("k_auto", "qc_threshold")]
    t0 = time.time()
    with mp.get_context("spawn").Pool(args.procs) as pool:
        res = pool.map(_task, tasks, chunksize=1)
    Js = {r[2] for r in res}
    if len(Js) != 1:
        raise SystemExit("the forward runs disagree on J: %s" % sorted(Js))
    out = {"workload": "single_bubble Float64 512x96, dt=2 s, ns=8, J = sum(prec * dx)",
           "steps": args.steps, "seed": args.seed, "dirs": args.dirs, "J": res[0][2],
           "directions": [{"dJ": r[3], "norm2_theta": r[4], "norm2_qv": r[5]} for r in res if r[0] == "dir"],
           "params": {r[1]: r[3] for r in res if r[0] == "param"},
           "generator": "tests/golden/make_tangent_single_bubble.py (oracle/oracle_tangent.cpp, forward mode)"}
    with open(OUT, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote %s in %.0f s" % (OUT, time.time() - t0))


if __name__ == "__main__":
    main()
