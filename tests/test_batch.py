"""Ensembles (moist_batch_*, model.Ensemble): members of different shapes advanced together give
each member's single-domain result bit for bit (which equals the oracle's), over calls of
different lengths (the launches of odd and even steps differ), in every precision mode; a NaN in
one member is reported for that member while the others finish their steps."""
import numpy as np
import pytest

from moist2d_b200 import abi, model
from moist2d_b200.init import sounding_bubbles
from oracle import bind
from states import compare, perturb, small_case

pytestmark = pytest.mark.gpu

MODES = [(np.float32, 0), (np.float32, abi.MOIST_FLAG_TRI_NATIVE), (np.float64, 0)]
IDS = ["f32-tri64", "f32-tri32", "f64"]


def members(T):
    out = []
    for j, (nx, nz) in enumerate([(96, 40), (33, 17), (64, 64), (130, 37)]):
        p, s = sounding_bubbles(T, nx=nx, nz=nz, nbub=1, seed=10 + j)
        perturb(s, p, 30 + j, wind=5.0, w=1.5)
        out.append((p, s))
    return out


@pytest.mark.parametrize("T,flags", MODES, ids=IDS)
def test_ensemble_matches_single_domains(T, flags):
    mem = members(T)
    with model.Ensemble([p for p, _ in mem], flags) as e:
        for i, (_, s) in enumerate(mem):
            e.upload(i, s)
        e.step(2)
        e.step(1)
        got = [e.download(i, s.copy()) for i, (_, s) in enumerate(mem)]
    for (p, s), g in zip(mem, got):
        ref = model.rk3_step(s.copy(), p, 3, flags=flags)
        compare(g, ref, p)
    p, s = mem[1]
    o = s.copy()
    bind.rk3_step(o, p, 3, tri64=(T == np.float32 and not flags))
    compare(got[1], o, p)


def test_ensemble_budget_and_member_access():
    mem = members(np.float32)
    with model.Ensemble([p for p, _ in mem]) as e:
        for i, (_, s) in enumerate(mem):
            e.upload(i, s)
        e.step(2)
        b = [e.budget(i) for i in range(len(mem))]
    for (p, s), bi in zip(mem, b):
        with model.Model(p) as m:
            m.upload(s)
            m.step(2)
            np.testing.assert_array_equal(m.budget(), bi)


def test_ensemble_nan_in_one_member():
    mem = members(np.float32)
    bad = mem[2][1]
    bad.rho_qv[5, 10] = np.float32(np.nan)
    with pytest.raises(FloatingPointError) as single:
        model.rk3_step(bad.copy(), mem[2][0], 2)
    with model.Ensemble([p for p, _ in mem]) as e:
        for i, (_, s) in enumerate(mem):
            e.upload(i, s)
        with pytest.raises(FloatingPointError) as ens:
            e.step(2)
        assert str(ens.value) == "member 2: " + str(single.value)
        assert e.nan_member == 2
        got = e.download(0, mem[0][1].copy())
    p0, s0 = mem[0]
    compare(got, model.rk3_step(s0.copy(), p0, 2), p0)


def test_ensemble_rejects_mixed_substeps():
    p1, _ = small_case(np.float32, 8, 6)
    p2 = p1.replace(ns=5)
    with pytest.raises(ValueError):
        model.Ensemble([p1, p2])


def test_member_stepped_alone_then_batch():
    """A member advanced through its own context (moist_batch_member + moist_rk3_step) swaps its
    State buffers; the next batch step continues from that State."""
    mem = members(np.float32)
    with model.Ensemble([p for p, _ in mem]) as e:
        for i, (_, s) in enumerate(mem):
            e.upload(i, s)
        e.step(1)
        ctx = e.member(2)
        model._raise(lib_step(ctx, 1), ctx, "moist_rk3_step on a member")
        e.step(2)
        got = [e.download(i, s.copy()) for i, (_, s) in enumerate(mem)]
    for j, ((p, s), g) in enumerate(zip(mem, got)):
        compare(g, model.rk3_step(s.copy(), p, 4 if j == 2 else 3), p)


def lib_step(ctx, n):
    from moist2d_b200._lib import lib
    return lib().moist_rk3_step(ctx, n)


@pytest.mark.parametrize("nthreads,tapes", [(0, 1), (0, 0), (3, -1)], ids=["packed", "packed-one-tape", "threads"])
@pytest.mark.parametrize("T", [np.float32, np.float64], ids=["f32", "f64"])
def test_batch_adjoint_matches_single_adjoints(T, nthreads, tapes):
    """moist_batch_adjoint_run gives every member the gradient of its own moist_adjoint_run
    (a context with the same streaming tracer sweep; the adjoint's atomic sums may round in a
    different order) and leaves the members where the batch continues from: with the members'
    kernels packed (a tape per step of a segment, or one tape and the segment's States; 3 steps
    in segments of 2 and 1) and with every member's own run from host threads."""
    mem = members(T)
    rng = np.random.default_rng(4)
    weights = []
    for p, _ in mem:
        w = np.zeros(p.ia)
        w[p.is_ - 1:p.ie] = float(p.dx)
        weights.append(w)
    seeds = [{"rho_theta": rng.standard_normal((p.ka, p.ia)) * 1e-3} for p, _ in mem]
    with model.Ensemble([p for p, _ in mem]) as e:
        for i, (_, s) in enumerate(mem):
            e.upload(i, s)
        e.set_adjoint_tapes(tapes)
        got = e.adjoint(3, 2, prec_weights=weights, state_seeds=seeds, nthreads=nthreads)
        e.step(1)
        fin = [e.download(i, s.copy()) for i, (_, s) in enumerate(mem)]
    for i, (p, s) in enumerate(mem):
        with model.Model(p, abi.MOIST_FLAG_TRACER_STREAM) as m:
            m.upload(s)
            ref = m.adjoint(3, 2, prec_weight=weights[i], state_seed=seeds[i])
        for f in abi.PROGNOSTIC:
            scale = max(np.max(np.abs(ref[f])), 1e-300)
            assert np.max(np.abs(got[i][f] - ref[f])) <= 1e-10 * scale, (i, f)
        for k in ("k_auto", "qc_threshold", "objective"):
            assert np.isclose(got[i][k], ref[k], rtol=1e-10, atol=0.0), (i, k)
        compare(fin[i], model.rk3_step(s.copy(), p, 4), p)
