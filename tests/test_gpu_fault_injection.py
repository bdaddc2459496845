"""GPU: host-side fault injection and request control, with no device fault.

wt_ctx_inject_alloc_failure fails the k-th device allocation from now with
WT_ENOMEM without calling cudaMalloc.  Every allocation of a solve's set-up and
first steps is failed in turn: the failing call raises WT_ENOMEM, the objects it
leaves are released to the context's device bytes before the attempt, and the
context then runs the solve to the same bits.  The serving engine keeps a
request whose admission failed at the head of its queue and serves it later; a
cancelled request releases its device memory at once; a preempted one resumes
from a host checkpoint (wt_state_checkpoint_*) to the bits of an uninterrupted
run.  The reference has none of this: a failed CuArray allocation ends its
evolve3d call with an exception (src/evolve.jl:1149-1358).
"""
import dataclasses
import gc

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _live(ctx):
    gc.collect()
    return ctx.memory()[0]


def _solve(wt, ctx, prec, made):
    g = wt.Mesh.uniform_hex(ctx, 8, 2, outer_tag=7, warp_A=0.05, precision=prec)
    made.append(g)
    c = wt.sample_background3d(g, wt.BG_ADM_PERTURBED, wt.workloads.adm_params(1))
    made.append(c)
    ws = wt.make_wave3d_workspace(g)
    made.append(ws)
    P, Q = g.zeros(), g.zeros()
    wt.initial_state(ws, wt.IC_GAUSSIANS, wt.gaussian_params(*wt.workloads.pulses(3, 1)), P, Q)
    wt.step_rk4_curved(P, Q, c, ws, 1e-3, 3, bc3d=wt.make_bc3d([2] * 6), metric=True)
    E = wt.wave3d_energy(P, Q, c, ws, metric=True)
    return P, Q, E


def _close(made):
    for o in reversed(made):
        o.close()
    made.clear()


@pytest.mark.parametrize("prec", [0, 1])
def test_every_allocation_failure_is_clean(wt, ctx, prec):
    import torch
    base = _live(ctx)
    made = []
    a0 = ctx.memory()[2]
    P0, Q0, E0 = _solve(wt, ctx, prec, made)
    n = ctx.memory()[2] - a0
    _close(made)
    assert _live(ctx) == base
    assert n >= 20, n                       # mesh, background, workspace and step buffers
    for k in range(n):
        ctx.inject_alloc_failure(k)
        with pytest.raises(wt.WaveToyError) as ei:
            _solve(wt, ctx, prec, made)
        assert ei.value.code == -3 and "injected" in str(ei.value), (k, str(ei.value))
        _close(made)
        assert _live(ctx) == base, k
    ctx.inject_alloc_failure(n)             # beyond this solve's allocations: never fires here
    P1, Q1, E1 = _solve(wt, ctx, prec, made)
    ctx.inject_alloc_failure(-1)
    assert torch.equal(P1, P0) and torch.equal(Q1, Q0) and E1 == E0
    _close(made)
    assert _live(ctx) == base and not ctx.nonfinite()


def _requests(wt):
    S = wt.serve
    specs = [(0, 3, 8, 24), (1, 2, 6, 20), (2, 2, 8, 16)]
    return [S.Request(rid=r, arrival=0.0, elements=e, n=n, steps=st, seed=700 + r, scale=0.5)
            for r, e, n, st in specs]


def _engine(wt, precision, **kw):
    return dict(hbm_budget=4e9, tick=4, precision=precision, keep_results=True, fill_nodes=None, **kw)


def _served_states(wt, ctx, precision, reqs, control=None):
    """Serve reqs on a fresh engine; control(eng, rids, round) runs before each poll."""
    S = wt.serve
    eng = wt.ServeEngine(ctx, wt.serve_desc(**_engine(wt, precision)))
    rids = [eng.submit(S.native_request(q)) for q in reqs]
    rnd = 0
    while eng.info()["waiting"] or eng.info()["active"]:
        if control:
            control(eng, rids, rnd)
        eng.poll()
        rnd += 1
    out = {}
    for rid in rids:
        if eng.status(rid)["status"] == wt.REQ_FINISHED:
            P, Q = eng.state(rid)
            out[rid] = (P.clone(), Q.clone(), eng.result(rid))
    return eng, rids, out


def test_serve_admission_retries_after_allocation_failure(wt, ctx):
    import torch
    S = wt.serve
    reqs = _requests(wt)[:1]
    base = _live(ctx)
    eng, _, ref = _served_states(wt, ctx, wt.WT_F64, reqs)
    eng.close()
    assert _live(ctx) == base
    # the allocations of the first round (admission, batch build)
    eng = wt.ServeEngine(ctx, wt.serve_desc(**_engine(wt, wt.WT_F64)))
    rid = eng.submit(S.native_request(reqs[0]))
    a0 = ctx.memory()[2]
    eng.poll()
    n = ctx.memory()[2] - a0
    eng.close()
    assert _live(ctx) == base and n >= 10
    for k in range(n):
        eng = wt.ServeEngine(ctx, wt.serve_desc(**_engine(wt, wt.WT_F64)))
        rid = eng.submit(S.native_request(reqs[0]))
        ctx.inject_alloc_failure(k)
        with pytest.raises(wt.WaveToyError) as ei:
            eng.poll()
        assert ei.value.code == -3, k
        st = eng.status(rid)
        assert st["status"] in (wt.REQ_WAITING, wt.REQ_RUNNING) and st["steps_left"] == reqs[0].steps, k
        eng.run()                            # retried: the request is served to the same bits
        P, Q = eng.state(rid)
        assert torch.equal(P, ref[0][0]) and torch.equal(Q, ref[0][1]), k
        eng.close()
        assert _live(ctx) == base, k


def test_serve_cancel_releases_at_once(wt, ctx):
    reqs = _requests(wt)
    base = _live(ctx)
    seen = {}

    def control(eng, rids, rnd):
        if rnd == 0:
            eng.cancel(rids[2])              # waiting: leaves the queue
            assert eng.status(rids[2])["status"] == wt.REQ_CANCELLED
        if rnd == 2:
            assert eng.status(rids[1])["status"] == wt.REQ_RUNNING
            before = _live(ctx)
            used = eng.info()["used_bytes"]
            eng.cancel(rids[1])              # running: leaves the batch, memory released now
            seen["freed"] = before - _live(ctx)
            seen["used"] = used - eng.info()["used_bytes"]
            st = eng.status(rids[1])
            assert st["status"] == wt.REQ_CANCELLED and 0 < st["steps_left"] < reqs[1].steps
            with pytest.raises(wt.WaveToyError):
                eng.cancel(rids[1])          # already cancelled

    eng, rids, out = _served_states(wt, ctx, wt.WT_F64, reqs, control)
    assert set(out) == {rids[0]} and eng.info()["done"] == 1
    assert seen["freed"] > 0 and seen["used"] > 0
    with pytest.raises(wt.WaveToyError):
        eng.cancel(rids[0])                  # finished
    with pytest.raises(wt.WaveToyError):
        eng.result(rids[1])                  # a cancelled request has no result
    eng.close()
    assert _live(ctx) == base


@pytest.mark.parametrize("precision", [0, 1])
def test_serve_preempted_request_resumes_bitwise(wt, ctx, precision):
    import torch
    reqs = _requests(wt)
    base = _live(ctx)
    eng, rids, ref = _served_states(wt, ctx, precision, reqs)
    eng.close()

    def control(eng, rids, rnd):
        if rnd == 2:
            used = eng.info()["used_bytes"]
            eng.preempt(rids[0])
            st = eng.status(rids[0])
            assert st["status"] == wt.REQ_PREEMPTED and st["preemptions"] == 1
            assert 0 < st["steps_left"] < reqs[0].steps
            assert eng.info()["used_bytes"] < used
            with pytest.raises(wt.WaveToyError):
                eng.preempt(rids[0])         # not running
        if rnd == 4 and eng.status(rids[1])["status"] == wt.REQ_RUNNING:
            eng.preempt(rids[1])

    eng, rids2, out = _served_states(wt, ctx, precision, reqs, control)
    assert set(out) == set(ref)
    assert eng.status(rids2[0])["preemptions"] == 1
    for rid in rids2:
        assert torch.equal(out[rid][0], ref[rid][0]) and torch.equal(out[rid][1], ref[rid][1]), rid
        assert out[rid][2]["dt"] == ref[rid][2]["dt"]
    eng.close()
    assert _live(ctx) == base and not ctx.nonfinite()


@pytest.mark.parametrize("prec", [0, 1])
def test_checkpoint_roundtrip_is_bitwise(wt, ctx, prec):
    import torch
    g = wt.Mesh.uniform_hex(ctx, 6, 3, periodic=True, warp_A=0.05, precision=prec)
    c = wt.sample_background3d(g, wt.BG_ADM_PERTURBED, wt.workloads.adm_params(2))
    ws = wt.make_wave3d_workspace(g)
    P, Q = g.zeros(), g.zeros()
    wt.initial_state(ws, wt.IC_GAUSSIANS, wt.gaussian_params(*wt.workloads.pulses(5, 2)), P, Q)
    dt = 0.2 * g.min_spacing() / wt.workloads.max_speed(wt.workloads.adm_params(2))
    wt.step_rk4_curved(P, Q, c, ws, dt, 5, metric=True)
    ck = wt.checkpoint_save(ws, P, Q)
    rs = 8 if prec == 0 else 4
    assert ck.size == g.nn * rs * (2 if prec == 0 else 4)
    wt.step_rk4_curved(P, Q, c, ws, dt, 7, metric=True)
    ws2 = wt.make_wave3d_workspace(g)        # another workspace, other state arrays
    P2, Q2 = g.zeros(), g.zeros()
    wt.checkpoint_load(ws2, P2, Q2, ck)
    wt.step_rk4_curved(P2, Q2, c, ws2, dt, 7, metric=True)
    assert torch.equal(P2, P) and torch.equal(Q2, Q)
    if prec == 1:                            # the FP32 low parts are part of the state
        half = g.nn * 8
        P3, Q3 = g.zeros(), g.zeros()
        wt.checkpoint_load(ws2, P3, Q3, np.concatenate([ck[:half], np.zeros(half, np.uint8)]))
        wt.step_rk4_curved(P3, Q3, c, ws2, dt, 7, metric=True)
        assert not torch.equal(P3, P)
    with pytest.raises(wt.WaveToyError):
        wt.checkpoint_load(ws2, P2, Q2, ck[:-1])


@pytest.mark.parametrize("preempt", [False, True])
def test_preemptive_admission(wt, ctx, preempt):
    """One slot (max_active = 1): a long request runs, a short one arrives.  With preemptive
    admission the long one is checkpointed, the short one runs and finishes first, and the
    long one resumes to the bits of its uninterrupted run; without it the short one waits."""
    import torch
    S = wt.serve
    long_q, short_q = _requests(wt)[0], _requests(wt)[1]
    long_q = dataclasses.replace(long_q, steps=60)
    short_q = dataclasses.replace(short_q, steps=8)
    alone = {}
    for q in (long_q, short_q):
        eng = wt.ServeEngine(ctx, wt.serve_desc(**_engine(wt, wt.WT_F64)))
        rid = eng.submit(S.native_request(q))
        eng.run()
        alone[q.rid] = tuple(t.clone() for t in eng.state(rid))
        eng.close()
    eng = wt.ServeEngine(ctx, wt.serve_desc(**_engine(wt, wt.WT_F64, max_active=1, preempt=preempt)))
    rl = eng.submit(S.native_request(long_q))
    eng.poll()
    eng.poll()
    rs = eng.submit(S.native_request(short_q))
    eng.run()
    L, Sh = eng.result(rl), eng.result(rs)
    if preempt:
        assert eng.status(rl)["preemptions"] == 1 and Sh["finished"] < L["finished"]
    else:
        assert eng.status(rl)["preemptions"] == 0 and Sh["admitted"] >= L["finished"]
    for rid, q in ((rl, long_q), (rs, short_q)):
        P, Q = eng.state(rid)
        assert torch.equal(P, alone[q.rid][0]) and torch.equal(Q, alone[q.rid][1]), (preempt, rid)
    eng.close()
