"""Served solves: requests that arrive while others run join the same batch;
every served result equals the same request stepped alone (<= 1e-6 relative
L2, FP32 state), and the split-precision results stay within 1e-5 of the
Float64 oracle."""
import dataclasses

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def requests(wt):
    S = wt.serve
    specs = [(0, 0.00, 3, 8, 40), (1, 0.00, 2, 6, 24), (2, 0.01, 2, 8, 60), (3, 0.02, 3, 6, 30),
             (4, 0.05, 2, 8, 20), (5, 0.05, 2, 6, 50)]
    return [S.Request(rid=r, arrival=t, elements=e, n=n, steps=st, seed=900 + r, scale=0.5 * (r % 3))
            for r, t, e, n, st in specs]


def test_served_results_equal_alone_and_oracle(wt, ctx, O):
    import torch
    S = wt.serve
    reqs = requests(wt)
    server = S.Server(ctx, precision=wt.WT_F32, hbm_budget=4e9, tick=8, keep_results=True)
    res = server.run(reqs)
    assert [r.rid for r in res] == [q.rid for q in reqs]
    # the work of several requests overlapped on the device
    assert any(a.admitted < b.finished and b.admitted < a.finished for a in res for b in res if a.rid < b.rid)
    for q, r in zip(reqs, res):
        mesh, coef, ws, Phi, Pi, dt = S.build_solve(ctx, q, wt.WT_F32, release=False)
        assert dt == r.dt
        wt.step_rk4_curved(Phi, Pi, coef, ws, dt, q.steps, bc3d=wt.make_bc3d([wt.BC_SOMMERFELD] * 6), metric=True)
        a = torch.cat([r.Phi, r.Pi]).double().cpu().numpy()
        b = torch.cat([Phi, Pi]).double().cpu().numpy()
        assert rel(a, b) <= 1e-6, q.rid
    for q, r in list(zip(reqs, res))[:2]:  # split-precision result against the Float64 oracle
        o = O.OracleMesh(q.n, q.elements, A=0.05, outer_tag=7)
        co = o.background(2, wt.workloads.adm_params(q.seed, q.scale))
        x, y, z = o.coords()
        c, amp, w = wt.workloads.pulses(q.seed, q.pulses, amp=(0.5, 1.0), width=(0.05, 0.15), centre=(0.25, 0.75))
        P0 = wt.workloads.gaussian_field(x, y, z, c, amp, w)
        Po, Qo = o.evolve_curved(co, P0, np.zeros_like(P0), r.dt, q.steps, bc=O.make_bc([2] * 6), use_metric=True)
        a = np.concatenate([r.Phi.double().cpu().numpy(), r.Pi.double().cpu().numpy()])
        assert rel(a, np.concatenate([Po, Qo])) <= 1e-5, q.rid


def test_server_admission_respects_budget(wt, ctx):
    S = wt.serve
    reqs = requests(wt)
    one = max(S.Server(ctx)._cost(q) for q in reqs)
    server = S.Server(ctx, precision=wt.WT_F32, hbm_budget=one * 1.01, tick=16)
    res = server.run(reqs)
    assert len(res) == len(reqs)
    assert server.peak_used <= server.budget
    cost = {q.rid: server._cost(q) for q in reqs}
    for a in res:  # requests that ran at the same time fit the budget together
        for b in res:
            if a.rid < b.rid and a.admitted < b.finished and b.admitted < a.finished:
                assert cost[a.rid] + cost[b.rid] <= server.budget
    # one slot: strictly one request at a time, all served
    res1 = S.Server(ctx, precision=wt.WT_F32, tick=16, max_active=1).run(reqs)
    spans = sorted((r.admitted, r.finished) for r in res1)
    assert len(res1) == len(reqs)
    assert all(spans[i][1] <= spans[i + 1][0] + 1e-9 for i in range(len(spans) - 1))
    with pytest.raises(ValueError):
        S.Server(ctx, hbm_budget=1e3).run(reqs[:1])


def test_engine_incremental_submission(wt, ctx):
    """The native engine used directly: two requests start, two more are submitted
    while they run (between polls) and join the same batch; every result equals
    the request stepped alone (FP64, <= 1e-12); the error paths leave it usable."""
    import dataclasses
    import torch
    S = wt.serve
    reqs = requests(wt)[:4]
    eng = wt.ServeEngine(ctx, wt.serve_desc(hbm_budget=4e9, tick=4, precision=wt.WT_F64, keep_results=True,
                                            fill_nodes=None))
    rids = [eng.submit(S.native_request(dataclasses.replace(q, arrival=0.0))) for q in reqs[:2]]
    with pytest.raises(wt.WaveToyError):          # not finished yet
        eng.result(rids[0])
    assert eng.poll() == 0 and eng.info()["active"] == 2
    eng.poll()
    rids += [eng.submit(S.native_request(dataclasses.replace(q, arrival=0.0))) for q in reqs[2:]]
    with pytest.raises(wt.WaveToyError):          # over the budget
        big = dataclasses.replace(reqs[0], elements=40)
        eng.submit(S.native_request(big, with_speed=False))
    eng.run()
    info = eng.info()
    assert info["done"] == 4 and info["active"] == 0 and info["waiting"] == 0 and info["used_bytes"] == 0
    res = [eng.result(r) for r in rids]
    assert min(r["admitted"] for r in res[2:]) > max(r["admitted"] for r in res[:2])
    assert any(b["admitted"] < a["finished"] for a in res[:2] for b in res[2:])   # joined running work
    for q, rid, r in zip(reqs, rids, res):
        assert r["precision"] == wt.WT_F64 and r["steps"] == q.steps and r["nodes"] == q.nodes
        Phi_s, Pi_s = eng.state(rid)
        mesh, coef, ws, Phi, Pi, dt = S.build_solve(ctx, q, wt.WT_F64, release=False)
        assert dt == r["dt"]
        wt.step_rk4_curved(Phi, Pi, coef, ws, dt, q.steps, bc3d=wt.make_bc3d([wt.BC_SOMMERFELD] * 6), metric=True)
        a = torch.cat([Phi_s, Pi_s]).cpu().numpy()
        b = torch.cat([Phi, Pi]).cpu().numpy()
        assert rel(a, b) <= 1e-12, q.rid
    eng.close()
    eng2 = wt.ServeEngine(ctx, wt.serve_desc(tick=8))
    rid = eng2.submit(S.native_request(dataclasses.replace(reqs[1], arrival=0.0)))
    eng2.run()
    with pytest.raises(wt.WaveToyError):          # no kept state without keep_results
        eng2.state(rid)
    eng2.close()
    assert not ctx.nonfinite()


@pytest.mark.parametrize("precision", [0, 1])
def test_engine_serves_time_dependent_background(wt, ctx, precision):
    """A sine-shift request (its background re-sampled at every RK4 stage inside the
    batch) served beside a static one: the result equals the same solve stepped alone
    (FP64 <= 1e-12, compensated FP32 <= 1e-6)."""
    import torch
    S = wt.serve
    bc = wt.make_bc3d([wt.BC_SOMMERFELD] * 6)
    c, a, w = wt.workloads.pulses(71, 2, amp=(0.5, 1.0), width=(0.08, 0.15))
    icp = wt.gaussian_params(c, a, w)
    A, t0, speed = 0.1, 0.02, 1.1 / 0.9
    q = wt.serve_request(0.0, 6, 2, warp_A=0.05, outer_tag=wt.SOMMERFELD_BDRY_TAG, bg_kind=wt.BG_SINE_SHIFT,
                         bg_params=(A, 1.0, t0), ic_params=icp, max_speed=speed, steps=9, bc3d=bc)
    eng = wt.ServeEngine(ctx, wt.serve_desc(hbm_budget=4e9, tick=4, precision=precision, keep_results=True,
                                            fill_nodes=None))
    rid = eng.submit(q)
    other = eng.submit(S.native_request(dataclasses.replace(requests(wt)[0], arrival=0.0)))
    eng.run()
    r = eng.result(rid)
    assert r["steps"] == 9 and eng.result(other)["steps"] > 0
    mesh = wt.Mesh.warped_uniform_hex(ctx, 6, 2, 0.0, 1.0, 0.05, outer_tag=wt.SOMMERFELD_BDRY_TAG,
                                      precision=precision)
    coef = wt.sample_background3d(mesh, wt.BG_SINE_SHIFT, (A, 1.0, t0))
    ws = wt.make_wave3d_workspace(mesh)
    Phi, Pi = mesh.zeros(), mesh.zeros()
    wt.initial_state(ws, wt.IC_GAUSSIANS, icp, Phi, Pi)
    dt = 0.2 * mesh.min_spacing() / speed
    assert abs(dt - r["dt"]) <= 1e-15 * dt
    wt.step_rk4_curved(Phi, Pi, coef, ws, r["dt"], 9, bc3d=bc, metric=True)
    Phi_s, Pi_s = eng.state(rid)
    got = torch.cat([Phi_s, Pi_s]).double().cpu().numpy()
    want = torch.cat([Phi, Pi]).double().cpu().numpy()
    assert rel(got, want) <= (1e-12 if precision == 0 else 1e-6)
    eng.close()
    assert not ctx.nonfinite()


def test_auto_precision_mixes_forms_in_one_batch(wt, ctx):
    """AUTO: requests with few steps run in FP32, the others in FP64, side by side in
    one batch; each result equals its request stepped alone in its form."""
    import dataclasses
    import torch
    S = wt.serve
    base = requests(wt)[:4]
    reqs = [dataclasses.replace(q, arrival=0.0, steps=st) for q, st in zip(base, (12, 30, 16, 28))]
    eng = wt.ServeEngine(ctx, wt.serve_desc(hbm_budget=4e9, tick=4, precision=wt.SERVE_AUTO,
                                            auto_fp32_max_steps=20, keep_results=True, fill_nodes=None))
    rids = [eng.submit(S.native_request(q)) for q in reqs]
    eng.run()
    res = [eng.result(r) for r in rids]
    assert [r["precision"] for r in res] == [wt.WT_F32, wt.WT_F64, wt.WT_F32, wt.WT_F64]
    assert max(r["admitted"] for r in res) < min(r["finished"] for r in res)   # all four ran together
    for q, rid, r in zip(reqs, rids, res):
        Phi_s, Pi_s = eng.state(rid)
        mesh, coef, ws, Phi, Pi, dt = S.build_solve(ctx, q, r["precision"], release=False)
        wt.step_rk4_curved(Phi, Pi, coef, ws, dt, q.steps, bc3d=wt.make_bc3d([wt.BC_SOMMERFELD] * 6), metric=True)
        tol = 1e-12 if r["precision"] == wt.WT_F64 else 1e-6
        a = torch.cat([Phi_s, Pi_s]).double().cpu().numpy()
        b = torch.cat([Phi, Pi]).double().cpu().numpy()
        assert rel(a, b) <= tol, q.rid
    eng.close()
