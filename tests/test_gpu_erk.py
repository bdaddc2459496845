"""GPU parity of the fixed-step Tsit5 (wt_step_erk_curved) against the oracle's:
static ADM and time-dependent gauge-wave backgrounds, Sommerfeld outer faces,
Kreiss-Oliger, the generic and the n = 8 kernels, steps launched one by one and
through the CUDA-graph replay (<= 1e-12 FP64, <= 1e-5 FP32); WT_ERK_RK4 is the
fused RK4 step."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.parametrize("N,prec,td,eps", [(6, 0, False, 0.1), (8, 0, False, 0.0), (6, 0, True, 0.0),
                                           (8, 1, False, 0.0)])
def test_tsit5_matches_oracle(wt, ctx, O, N, prec, td, eps):
    import torch
    g = wt.Mesh.uniform_hex(ctx, N, 2, outer_tag=7, warp_A=0.05, precision=prec)
    o = O.OracleMesh(N, 2, A=0.05, outer_tag=7)
    p = wt.workloads.adm_params(5)
    if td:
        c, co, tdb = wt.sample_background3d(g, wt.BG_GAUGE_WAVE, (0.2, 1.0, 0.1)), None, (4, (0.2, 1.0), 0.1)
    else:
        c, co, tdb = wt.sample_background3d(g, wt.BG_ADM_PERTURBED, p), o.background(2, p), None
    ws = wt.make_wave3d_workspace(g)
    x, y, z = o.coords()
    P0 = np.sin(2 * np.pi * x) * np.cos(np.pi * (y - z))
    Q0 = 0.3 * np.cos(np.pi * (x + 2 * z))
    dt = 0.2 * o.min_spacing() / (1.0 if td else wt.workloads.max_speed(p))
    dty = torch.float64 if prec == 0 else torch.float32
    P = torch.tensor(P0, dtype=dty, device="cuda")
    Q = torch.tensor(Q0, dtype=dty, device="cuda")
    bc = wt.make_bc3d([2] * 6)
    wt.step_erk_curved(P, Q, c, ws, dt, 2, wt.ERK_TSIT5, eps_KO=eps, bc3d=bc, metric=True)
    wt.step_erk_curved(P, Q, c, ws, dt, 5, wt.ERK_TSIT5, eps_KO=eps, bc3d=bc, metric=True)
    Po, Qo = o.evolve_curved_erk(co, P0, Q0, dt, 7, method=1, eps_ko=eps, bc=O.make_bc([2] * 6), use_metric=True,
                                 td=tdb)
    tol = 1e-12 if prec == 0 else 1e-5
    assert rel(P.double().cpu().numpy(), Po) < tol and rel(Q.double().cpu().numpy(), Qo) < tol
    if td:
        assert abs(c.time - (0.1 + 7 * dt)) < 1e-14
    assert not ctx.nonfinite()


def test_erk_rk4_is_the_fused_step(wt, ctx):
    import torch
    g = wt.Mesh.uniform_hex(ctx, 5, 2, outer_tag=7, warp_A=0.05)
    c = wt.sample_background3d(g, wt.BG_ADM_PERTURBED, wt.workloads.adm_params(2))
    ws = wt.make_wave3d_workspace(g)
    P = torch.randn(g.nn, dtype=torch.float64, device="cuda")
    Q = torch.randn(g.nn, dtype=torch.float64, device="cuda")
    P2, Q2 = P.clone(), Q.clone()
    bc = wt.make_bc3d([2] * 6)
    wt.step_erk_curved(P, Q, c, ws, 1e-3, 4, wt.ERK_RK4, bc3d=bc, metric=True)
    wt.step_rk4_curved(P2, Q2, c, ws, 1e-3, 4, bc3d=bc, metric=True)
    assert torch.equal(P, P2) and torch.equal(Q, Q2)
    with pytest.raises(wt.WaveToyError):
        wt.step_erk_curved(P, Q, c, ws, 1e-3, 1, 7)


def test_caller_tableau(wt, ctx, O):
    """wt_step_erk_curved_tableau: Tsit5's own tableau gives the built-in method's bits; a
    12-stage method (three RK4 steps of dt/3 as one tableau, more slopes than the built-in
    methods use) equals the oracle's RK4 at dt/3; a non-explicit or oversized tableau is
    refused."""
    import torch
    g = wt.Mesh.uniform_hex(ctx, 6, 2, outer_tag=7, warp_A=0.05)
    o = O.OracleMesh(6, 2, A=0.05, outer_tag=7)
    p = wt.workloads.adm_params(5)
    c, co = wt.sample_background3d(g, wt.BG_ADM_PERTURBED, p), o.background(2, p)
    ws = wt.make_wave3d_workspace(g)
    x, y, z = o.coords()
    P0 = np.sin(2 * np.pi * x) * np.cos(np.pi * (y - z))
    Q0 = 0.3 * np.cos(np.pi * (x + 2 * z))
    dt = 0.2 * o.min_spacing() / wt.workloads.max_speed(p)
    bc = wt.make_bc3d([2] * 6)
    P1, Q1 = torch.tensor(P0, device="cuda"), torch.tensor(Q0, device="cuda")
    P2, Q2 = P1.clone(), Q1.clone()
    wt.step_erk_curved(P1, Q1, c, ws, dt, 4, wt.ERK_TSIT5, bc3d=bc, metric=True)
    wt.step_erk_curved_tableau(P2, Q2, c, ws, dt, 4, *wt.erk_tableau(wt.ERK_TSIT5), bc3d=bc, metric=True)
    assert torch.equal(P1, P2) and torch.equal(Q1, Q2)
    C2, A2, B2 = wt.composed_tableau(*wt.erk_tableau(wt.ERK_RK4), 3)
    P3, Q3 = torch.tensor(P0, device="cuda"), torch.tensor(Q0, device="cuda")
    wt.step_erk_curved_tableau(P3, Q3, c, ws, dt, 5, C2, A2, B2, bc3d=bc, metric=True)
    Po, Qo = o.evolve_curved(co, P0, Q0, dt / 3, 15, bc=O.make_bc([2] * 6), use_metric=True)
    assert rel(P3.cpu().numpy(), Po) < 1e-12 and rel(Q3.cpu().numpy(), Qo) < 1e-12
    bad = A2.copy()
    bad[3, 5] = 0.1                                   # an implicit coupling
    with pytest.raises(wt.WaveToyError):
        wt.step_erk_curved_tableau(P3, Q3, c, ws, dt, 1, C2, bad, B2, bc3d=bc, metric=True)
    C4, A4, B4 = wt.composed_tableau(*wt.erk_tableau(wt.ERK_RK4), 5)   # 20 stages
    with pytest.raises(wt.WaveToyError):
        wt.step_erk_curved_tableau(P3, Q3, c, ws, dt, 1, C4, A4, B4, bc3d=bc, metric=True)
    assert not ctx.nonfinite()
