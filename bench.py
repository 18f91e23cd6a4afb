#!/usr/bin/env python
"""Benchmark of the large time step (rk3_step!) on B200: cell-steps/s.

One step = one large step (rk3_step!, moist.jl:1589) of the whole domain; one cell-step = one
interior cell advanced by one large step. Default workload: the 2048 x 128 analytic-sounding
domain with five seeded warm bubbles (dx = 250 m, dz = 125 m, dt = 2 s, ns = 8), Float32
state with FP64 w-p elimination, synthetic seeded input.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload plain|bubble] [--precision f32|f64]

value:  device time of K steps (CUDA events on the context stream around each step, L2 flushed
        by a 256 MiB write before every timed step), max over ranks, cells x K x N / time. Each
        timed step is followed by a profiled step (events at every change of kernel group: they
        cost the stream several microseconds each, so they are kept out of the value).
e2e:    the same metric through the reference-facing call rk3_step!(s, p) on a host State
        (moist_rk3_step_host: upload, step, download every step, page-locked host arrays),
        wall clock around each call.
roofline: the kernel group with the largest device time; achieved = its algorithmic bytes per
        launch (words per cell below x cells) / its mean launch time in the profiled steps.
adjoint: (1 GPU, Float32) moist_adjoint_run on the 512 x 96 single-bubble domain, 600 steps,
        rain objective, checkpoints every 50 steps: forward and reverse wall times and their ratio.
adjoint_ensemble: (1 GPU, Float32) moist_batch_adjoint_run on 64 uneven members (nx 512..1536,
        nz 96/128), 20 steps, the members' kernels packed against every member's own
        moist_adjoint_run from a host thread.
ensemble: (1 GPU, Float32) the batched forward: 256 uneven members advanced together (one packed
        launch per kernel of the step, one CUDA graph per step), device time per step, its
        cell-steps/s, HBM fraction of the whole step's algorithmic bytes and ratio to `value`.
Multi-GPU: independent replicas (the domain does not shard; ensemble members would).
"""
import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "cell-steps/s on 1 B200: batched/adjoint vs plain fwd at FP64-tol; HBM % of peak"

# algorithmic words per cell per launch of each kernel group (1 word = sizeof(T)): the unique
# inter-phase field traffic of the reference algorithm, W(ns) = 10 + sum_stages(50 + 20 m_s)
GROUPS = ("physics", "prologue", "substep", "tracer", "update", "other")
WORDS = {"physics": 10, "prologue": 23, "substep": 20, "tracer": 16, "update": 11, "other": 0}


def words_per_cell_step(ns):
    ms = (max(1, -(-ns // 3)), max(1, -(-ns // 2)), ns)
    return 10 + sum(50 + 20 * m for m in ms)


def group_instances(ns):
    """Launch instances of each group per large step."""
    ms = (max(1, -(-ns // 3)), max(1, -(-ns // 2)), ns)
    return {"physics": 1, "prologue": 3, "substep": sum(ms), "tracer": 3, "update": 3, "other": 1}


def make_workload(name, T):
    from moist2d_b200.init import sounding_bubbles, warm_bubble
    if name == "plain":
        p, s = sounding_bubbles(T)
        desc = ("plain forward, 2048x128 cells (dx=250 m, dz=125 m), analytic sounding + 5 seeded "
                "warm bubbles, dt=2 s, ns=8")
    elif name == "bubble":
        p, s = warm_bubble(T)
        desc = "warm moist bubble, 200x100 cells of 100 m, dt=1 s, ns=6"
    else:
        raise SystemExit("unknown workload " + name)
    return p, s, desc


def max_over_ranks(x, world, device="cuda"):
    """The largest x over the ranks: a replicated job takes as long as its slowest rank."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(cells, world, seconds):
    """Whole-job cell-steps/s of `world` replicas of `cells` cells, one step per `seconds`."""
    return cells * world / seconds


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ncu_traffic(workload, precision):
    """DRAM bytes per launch of each kernel group from a committed ncu capture, if any."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(path):
        return {}
    with open(path) as f:
        d = json.load(f)
    return d.get("%s-%s" % (workload, precision), {})


class Clocks:
    """nvidia-smi clock / throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        sm, mx, reasons = [], None, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_baseline(workload, T, budget_s=12.0, max_steps=40):
    """The oracle's threaded build timed on the host cores on a bounded sample of the workload."""
    from oracle import bind  # builds the oracle if needed
    so = os.path.join(ROOT, "oracle", "libmoist_oracle_omp.so")
    if not os.path.exists(so):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)
    L = C.CDLL(so)
    p, s, _ = make_workload(workload, T)
    cp = p.to_c()
    h = s.to_c()
    cells = p.Nx * p.Nz
    L.oracle_rk3_step(C.byref(cp), p.precision, 1, C.byref(h), 1)  # warm-up step
    n, t0 = 0, time.perf_counter()
    while n < max_steps and time.perf_counter() - t0 < budget_s:
        L.oracle_rk3_step(C.byref(cp), p.precision, 1, C.byref(h), 1)
        n += 1
    dt = time.perf_counter() - t0
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    out = {"value": cells * n / dt, "unit": "cell-steps/s", "cores": cores, "kind": "port",
           "sample": "%d large steps of the %dx%d domain after 1 warm-up step (%.1f s), threaded "
                     "C++ restatement of rk3_step! (OpenMP over columns)" % (n, p.Nx, p.Nz, dt)}
    # one thread in the reference's loop order (the serial oracle, JULIA_NUM_THREADS=1)
    L1 = bind.lib()
    p, s, _ = make_workload(workload, T)
    cp = p.to_c()
    h = s.to_c()
    L1.oracle_rk3_step(C.byref(cp), p.precision, 1, C.byref(h), 1)
    n1, t1 = 0, time.perf_counter()
    while n1 < max_steps and time.perf_counter() - t1 < budget_s / 2:
        L1.oracle_rk3_step(C.byref(cp), p.precision, 1, C.byref(h), 1)
        n1 += 1
    dt1 = time.perf_counter() - t1
    out["single_thread"] = {"value": cells * n1 / dt1, "unit": "cell-steps/s", "cores": 1,
                            "sample": "%d large steps after 1 warm-up step (%.1f s), serial C++ "
                                      "restatement in the reference's loop order" % (n1, dt1)}
    return out


def measure_ensemble(nmem, steps, warmup, peak, plain_value):
    """Ensemble of nmem uneven Float32 members (nx in {256, ..., 2048}, nz in {64, 96, 128},
    seeded bubbles on the analytic sounding), one packed launch per kernel of the step for all
    members, each step one CUDA graph; device time of `steps` steps from CUDA events. The
    members' fields (113 MB each for 256 members) exceed L2, so no flush is needed."""
    from moist2d_b200 import model
    from moist2d_b200.init import ensemble_member
    t0 = time.perf_counter()
    mem = [ensemble_member(np.float32, member=m) for m in range(nmem)]
    cells = sum(p.Nx * p.Nz for p, _ in mem)
    words = words_per_cell_step(mem[0][0].ns)
    with model.Ensemble([p for p, _ in mem]) as e:
        for i, (_, s) in enumerate(mem):
            e.upload(i, s)
        setup_s = time.perf_counter() - t0
        tune = e.autotune(2)
        e.step(warmup)
        ms = e.time_steps(steps) / steps
        tot, g = e.profile(2)
    value = cells / (ms / 1e3)
    # each group's algorithmic bytes per step (WORDS per cell and launch x launches per step)
    # over its device time, against the measured HBM copy bandwidth
    inst = group_instances(mem[0][0].ns)
    group_frac = {}
    for k, x in zip(GROUPS, g):
        gms = float(x) / 2
        if WORDS[k] and gms > 0:
            group_frac[k] = WORDS[k] * 4 * cells * inst[k] / (gms / 1e3) / 1e9 / peak
    one = one_domain_per_launch(mem)
    return {"members": nmem, "cells": cells, "steps": steps, "warmup": warmup, "ms_per_step": ms,
            "value": value, "unit": "cell-steps/s", "vs_plain": value / plain_value,
            "one_domain_per_launch": one, "vs_one_domain_per_launch": one["ms_per_step"] / ms,
            "hbm_frac": cells * words * 4 / (ms / 1e3) / 1e9 / peak,
            "group_ms_per_step": {k: float(x) / 2 for k, x in zip(GROUPS, g)},
            "group_hbm_frac": group_frac,
            "setup_s": setup_s, "autotune": tune,
            "workload": "%d members, nx in {256,...,2048}, nz in {64,96,128}, dx=250 m, dz=125 m, "
                        "dt=2 s, ns=8, one seeded bubble each on the analytic sounding, Float32 "
                        "state with fp64 w-p elimination" % nmem}


def one_domain_per_launch(mem, steps=3):
    """The ensemble's members advanced the plain way, one domain per launch: each member in its
    own context (its own kernels, autotuned like the single-domain workload), one member after
    the other; the device time of a large step of every member, summed over the members."""
    from moist2d_b200 import model
    total = 0.0
    for p, s in mem:
        with model.Model(p) as m:
            m.upload(s)
            m.autotune(1)
            m.time_steps(1)  # warm-up
            total += m.time_steps(steps) / steps
    cells = sum(p.Nx * p.Nz for p, _ in mem)
    return {"ms_per_step": total, "value": cells / (total / 1e3), "unit": "cell-steps/s",
            "how": "each member in its own context (single-domain kernels, autotuned), members one "
                   "after the other, device time of %d large steps per member (CUDA events), "
                   "summed" % steps}


def measure_adjoint(nsteps, ckpt):
    """Adjoint workload: 512 x 96 single bubble, Float32 forward, objective = total surface rain
    after nsteps large steps, gradient w.r.t. the initial State and K_auto, Qc_threshold through
    moist_adjoint_run with checkpoints every ckpt steps. Wall time of the forward run and of the
    reverse sweep (recomputation included), both measured by the library around synchronised
    device work."""
    from moist2d_b200 import model
    from moist2d_b200.init import single_bubble
    p, s = single_bubble(np.float32)
    w = np.zeros(p.ia)
    w[p.is_ - 1:p.ie] = float(p.dx)
    with model.Model(p) as m:
        m.upload(s)
        m.adjoint(2, 1, prec_weight=w)  # warm-up: allocation of the adjoint buffers
        m.upload(s)
        g = m.adjoint(nsteps, ckpt, prec_weight=w)
    cells = p.Nx * p.Nz
    return {"workload": "single bubble 512x96 (dx=250 m, dz=125 m), dt=2 s, ns=8, Float32 state, "
                        "rain objective, gradient w.r.t. the initial State, K_auto, Qc_threshold",
            "steps": nsteps, "ckpt_every": ckpt, "forward_ms": g["forward_ms"], "reverse_ms": g["reverse_ms"],
            "adjoint_over_forward": g["reverse_ms"] / g["forward_ms"],
            "forward_cell_steps_per_s": cells * nsteps / (g["forward_ms"] / 1e3),
            "adjoint_cell_steps_per_s": cells * nsteps / (g["reverse_ms"] / 1e3),
            "objective": g["objective"], "dJ_dK_auto": g["k_auto"], "dJ_dQc_threshold": g["qc_threshold"]}


def measure_adjoint_ensemble(nmem, nsteps, ckpt):
    """Batched adjoint: nmem Float32 members (nx in {512, 1024, 1536}, nz in {96, 128}, seeded
    bubbles on the analytic sounding), rain objective per member, moist_batch_adjoint_run over
    nsteps large steps with checkpoints every ckpt steps: wall time with the members' kernels
    packed (nthreads = 0, one launch per kernel for all members) and with every member's own
    moist_adjoint_run from nmem host threads, and the batched forward's device time for the same
    steps."""
    from moist2d_b200 import model
    from moist2d_b200.init import ensemble_member
    mem = [ensemble_member(np.float32, seed=5, member=m, nx_choices=(512, 1024, 1536), nz_choices=(96, 128))
           for m in range(nmem)]
    cells = sum(p.Nx * p.Nz for p, _ in mem)
    weights = []
    for p, _ in mem:
        w = np.zeros(p.ia)
        w[p.is_ - 1:p.ie] = float(p.dx)
        weights.append(w)
    out = {"members": nmem, "cells": cells, "steps": nsteps, "ckpt_every": ckpt}
    with model.Ensemble([p for p, _ in mem]) as e:
        def upload():
            for i, (_, s) in enumerate(mem):
                e.upload(i, s)
        upload()
        e.adjoint(ckpt, ckpt, prec_weights=weights)  # warm-up: the members' adjoint buffers
        for name, nt in (("packed", 0), ("member_threads", nmem)):
            upload()
            t0 = time.perf_counter()
            g = e.adjoint(nsteps, ckpt, prec_weights=weights, nthreads=nt)
            out[name + "_ms"] = (time.perf_counter() - t0) * 1e3
            if nt == 0:
                out["packed_forward_ms"] = g[0]["forward_ms"]
                out["packed_reverse_ms"] = g[0]["reverse_ms"]
        upload()
        e.step(2)
        out["forward_batched_ms"] = e.time_steps(nsteps)
    out["speedup_vs_member_threads"] = out["member_threads_ms"] / out["packed_ms"]
    out["adjoint_cell_steps_per_s"] = cells * nsteps / (out["packed_ms"] / 1e3)
    out["adjoint_over_batched_forward"] = out["packed_ms"] / out["forward_batched_ms"]
    out["workload"] = ("%d members, nx in {512,1024,1536}, nz in {96,128}, dx=250 m, dz=125 m, dt=2 s, ns=8, "
                       "Float32, rain objective per member, %d of the 900 steps" % (nmem, nsteps))
    return out


def run_reference(args, rank, world):
    """--impl reference: the reference's CPU path (no Julia here: the threaded oracle port)."""
    if rank != 0:
        return
    T = np.float32 if args.precision == "f32" else np.float64
    from oracle import bind  # noqa: F401
    so = os.path.join(ROOT, "oracle", "libmoist_oracle_omp.so")
    if not os.path.exists(so):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)
    L = C.CDLL(so)
    p, s, desc = make_workload(args.workload, T)
    cp = p.to_c()
    h = s.to_c()
    cells = p.Nx * p.Nz
    for _ in range(args.warmup):
        L.oracle_rk3_step(C.byref(cp), p.precision, 1, C.byref(h), 1)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        L.oracle_rk3_step(C.byref(cp), p.precision, 1, C.byref(h), 1)
    dt = time.perf_counter() - t0
    value = cells * args.steps / dt
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "cell-steps/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": dt * 1e3 / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": args.precision, "data": "synthetic",
            "config": {"workload": desc, "cells": cells,
                       "reference": "Julia moist.jl is not runnable here (no Julia toolchain); "
                                    "its CPU path is timed as the threaded C++ restatement"},
            "cpu_baseline": {"value": value, "unit": "cell-steps/s", "kind": "port", "cores": cores,
                             "sample": "%d timed large steps of the full domain after %d warm-up "
                                       "steps" % (args.steps, args.warmup)},
            "e2e": {"value": value, "unit": "cell-steps/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=("ours", "reference"))
    ap.add_argument("--workload", default="plain", choices=("plain", "bubble"))
    ap.add_argument("--precision", default="f32", choices=("f32", "f64"))
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end measurement")
    ap.add_argument("--ensemble", type=int, default=256,
                    help="members of the batched-ensemble measurement (0 skips it)")
    ap.add_argument("--adjoint-steps", type=int, default=600,
                    help="large steps of the adjoint measurement (0 skips it)")
    ap.add_argument("--adjoint-ensemble", type=int, default=64,
                    help="members of the batched-adjoint measurement (0 skips it)")
    args = ap.parse_args()
    if args.warmup < 3:
        raise SystemExit("--warmup must be >= 3")

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    import torch
    import torch.distributed as dist

    torch.cuda.set_device(local_rank)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))

    from moist2d_b200 import _lib, abi
    from moist2d_b200.model import Model, _raise
    L = _lib.lib()
    _raise(L.moist_set_device(local_rank), None, "moist_set_device")

    T = np.float32 if args.precision == "f32" else np.float64
    p, s, desc = make_workload(args.workload, T)
    cells = p.Nx * p.Nz
    bpw = np.dtype(T).itemsize
    m = Model(p)
    m.upload(s)
    tune = m.autotune(3)  # strip width and tracer sweep; leaves the State as it was
    ext = torch.cuda.ExternalStream(L.moist_stream(m.ctx), device=torch.device("cuda", local_rank))
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    total = C.c_float()
    gms = (C.c_float * abi.MOIST_NGROUPS)()
    gl = (C.c_longlong * abi.MOIST_NGROUPS)()

    for _ in range(args.warmup):
        _raise(L.moist_step_profile(m.ctx, 1, C.byref(total), gms, gl), m.ctx, "warm-up step")

    # the end-to-end leg below replays the timed stretch of simulated time: a page-locked host
    # State holding the State the timed steps start from
    h = None
    if not args.no_e2e:
        ia, ka = p.ia, p.ka
        fields = ("rho", "rho_u", "rho_w", "rho_theta", "rho_qv", "rho_qc", "rho_qr")
        tdt = torch.float32 if T is np.float32 else torch.float64
        pinned = {}
        for f in fields:
            a = torch.empty((ia, ka), dtype=tdt, pin_memory=True).numpy().T  # (ka, ia) column-major
            a[...] = getattr(s, f)
            pinned[f] = a
        prec = torch.zeros(ia, dtype=tdt, pin_memory=True).numpy()
        h = abi.moist_state_host()
        for f in fields:
            setattr(h, f, pinned[f].ctypes.data)
        h.prec = prec.ctypes.data
        nbytes = (len(fields) * ka * ia + ia) * bpw
        _raise(L.moist_download_state(m.ctx, C.byref(h)), m.ctx, "e2e start state")

    clocks = Clocks(local_rank)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    # K plain steps, each between its own two CUDA events, give the value; each is followed by a
    # profiled step (an event at every change of kernel group) for the per-group split and the
    # roofline. The group events cost the stream several microseconds each, so they stay out of
    # the value; alternating the two samples the same stretch of simulated time.
    step_ms = 0.0
    prof_ms = 0.0
    one = C.c_float()
    group_ms = np.zeros(abi.MOIST_NGROUPS)
    launches = np.zeros(abi.MOIST_NGROUPS, dtype=np.int64)
    for _ in range(args.steps):
        with torch.cuda.stream(ext):
            flush.zero_()  # evict L2 (126 MB) before the step
        _raise(L.moist_time_steps(m.ctx, 1, C.byref(one)), m.ctx, "timed step")
        step_ms += one.value
        with torch.cuda.stream(ext):
            flush.zero_()
        _raise(L.moist_step_profile(m.ctx, 1, C.byref(total), gms, gl), m.ctx, "profiled step")
        prof_ms += total.value
        group_ms += np.array(gms[:])
        launches += np.array(gl[:])
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clk = clocks.stop()

    t_max = max_over_ranks(step_ms / args.steps, world)
    value = job_throughput(cells, world, t_max / 1e3)

    # end to end: rk3_step!(s, p) on a page-locked host State, every step, over the same 2K steps
    # of simulated time as the timed region (the step's cost changes as the bubbles develop)
    e2e = None
    if h is not None:
        for _ in range(2):  # upload and download only: the call path warmed, the State unchanged
            _raise(L.moist_rk3_step_host(m.ctx, C.byref(h), 0), m.ctx, "e2e warm-up")
        ne2e = 2 * args.steps
        if world > 1:
            dist.barrier()
        t0 = time.perf_counter()
        for _ in range(ne2e):
            _raise(L.moist_rk3_step_host(m.ctx, C.byref(h), 1), m.ctx, "e2e step")
        te = max_over_ranks((time.perf_counter() - t0) / ne2e, world)
        e2e = {"value": job_throughput(cells, world, te), "unit": "cell-steps/s", "h2d_bytes_per_step": nbytes,
               "d2h_bytes_per_step": nbytes, "ms_per_step": te * 1e3, "steps": ne2e,
               "how": "moist_rk3_step_host: H2D of the 7 prognostic fields + prec from page-locked "
                      "memory, one rk3 step, D2H of the same, wall clock per call; the calls start "
                      "from the State the timed region started from and advance the same 2K steps"}

    # roofline of the dominant kernel group, from the events of the timed region
    inst = group_instances(p.ns)
    gnames = GROUPS
    gi = int(np.argmax(group_ms))
    gname = gnames[gi]
    n_inst = inst[gname] * args.steps
    mean_ms = group_ms[gi] / n_inst
    alg_bytes = WORDS[gname] * bpw * cells
    achieved = alg_bytes / (mean_ms / 1e3) / 1e9
    peak, peak_kind = measured_peaks()
    traffic = ncu_traffic(args.workload, args.precision).get(gname)
    roofline = {"bound": "hbm", "kernel": gname, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": traffic,
                "algorithmic_bytes_per_launch": alg_bytes, "mean_launch_ms": mean_ms,
                "peak_kind": peak_kind,
                "step_frac": cells * words_per_cell_step(p.ns) * bpw / (t_max / 1e3) / 1e9 / peak}

    m.close()
    ens = None
    if rank == 0 and world == 1 and args.ensemble > 0 and args.precision == "f32":
        try:
            ens = measure_ensemble(args.ensemble, max(3, min(args.steps, 10)), args.warmup, peak, value)
        except Exception as e:  # the ensemble must not hide the single-domain number
            ens = {"value": None, "error": str(e)}
    adj = None
    if rank == 0 and world == 1 and args.adjoint_steps > 0 and args.precision == "f32":
        try:
            adj = measure_adjoint(args.adjoint_steps, 50)
        except Exception as e:
            adj = {"error": str(e)}
    adj_ens = None
    if rank == 0 and world == 1 and args.adjoint_ensemble > 0 and args.precision == "f32":
        try:
            adj_ens = measure_adjoint_ensemble(args.adjoint_ensemble, 20, 10)
        except Exception as e:
            adj_ens = {"error": str(e)}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        try:
            cpu = cpu_baseline(args.workload, T)
        except Exception as e:  # a baseline failure must not hide the GPU number
            cpu = {"value": None, "error": str(e)}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "cell-steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_max,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": args.precision, "data": "synthetic",
            "config": {"workload": desc, "cells": cells, "precision": args.precision +
                       (" state, fp64 w-p elimination" if args.precision == "f32" else ""),
                       "l2": "flushed before every timed step (256 MiB write)",
                       "timing": "K plain steps (CUDA events around each) give value and ms_per_step; "
                                 "each is followed by a profiled step (CUDA events at every change of "
                                 "kernel group) that gives kernel_ms_per_step and the roofline; "
                                 "gpu_launches counts the launches of all 2K steps",
                       "parallelism": "replicas" if world > 1 else "single domain",
                       "words_per_cell_step": words_per_cell_step(p.ns), "autotune": tune},
            "roofline": roofline,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": 2 * int(launches.sum()),
            "kernel_ms_per_step": {g: float(group_ms[j] / args.steps) for j, g in enumerate(gnames)},
            "profiled_ms_per_step": prof_ms / args.steps,
            "clocks": clk,
            "ensemble": ens,
            "adjoint": adj,
            "adjoint_ensemble": adj_ens,
        }
        print(json.dumps(line), flush=True)

    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
