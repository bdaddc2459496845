"""GPU parity of the time-dependent (spacetime-metric) backgrounds,
MetricBackground3D with the gauge wave / sine shift (src/wave3d_curved.jl:56-71):
coefficients sampled at a time t against the oracle's 3+1 split, RK4 with the
background re-sampled at every stage time (src/evolve.jl:1287-1307) against the
oracle's stage-resampled RK4 (<= 1e-12 FP64, <= 1e-5 FP32), the coefficients'
time advancing with the steps (also through the CUDA-graph replay), and the
exact plane-wave solution on the periodic cube."""
import numpy as np
import pytest

from test_oracle_metric_bg import exact

pytestmark = pytest.mark.gpu


def rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.parametrize("kind", [4, 5])
def test_sampled_at_time_matches_oracle(wt, ctx, O, kind):
    g = wt.Mesh.uniform_hex(ctx, 5, 3, periodic=True)
    o = O.OracleMesh(5, 3, periodic=True)
    c = wt.sample_background3d(g, kind, (0.2, 1.0, 0.1))
    assert c.time == 0.1
    assert rel(c.get(), o.background(kind, [0.2, 1.0, 0.1])) < 1e-14
    c.set_time(0.73)
    assert c.time == 0.73
    assert rel(c.get(), o.background(kind, [0.2, 1.0, 0.73])) < 1e-14
    static = wt.sample_background3d(g, wt.BG_MINKOWSKI)
    with pytest.raises(wt.WaveToyError):
        static.set_time(1.0)
    with pytest.raises(wt.WaveToyError):
        wt.sample_background3d(g, kind, (1.5, 1.0, 0.0))


@pytest.mark.parametrize("kind,N,M,prec", [(4, 6, 2, 0), (5, 6, 2, 0), (4, 8, 2, 0), (5, 8, 2, 1)])
def test_stage_resampled_rk4_matches_oracle(wt, ctx, O, kind, N, M, prec):
    """Warped mesh, Sommerfeld outer faces, metric terms on: 2 steps launched one by one,
    then 8 through the graph replay; the coefficients end at t0 + 10 dt."""
    import torch
    A, d, t0 = 0.15, 1.0, 0.05
    g = wt.Mesh.uniform_hex(ctx, N, M, outer_tag=7, warp_A=0.05, precision=prec)
    o = O.OracleMesh(N, M, A=0.05, outer_tag=7)
    c = wt.sample_background3d(g, kind, (A, d, t0))
    ws = wt.make_wave3d_workspace(g)
    x, y, z = o.coords()
    P0 = np.sin(2 * np.pi * x) * np.cos(np.pi * y) * np.sin(np.pi * z + 0.3)
    Q0 = 0.5 * np.cos(2 * np.pi * (x + y))
    speed = 1.0 if kind == 4 else (1 + A) / (1 - A)
    dt = 0.2 * o.min_spacing() / speed
    dty = torch.float64 if prec == 0 else torch.float32
    P = torch.tensor(P0, dtype=dty, device="cuda")
    Q = torch.tensor(Q0, dtype=dty, device="cuda")
    bc = wt.make_bc3d([2] * 6)
    wt.step_rk4_curved(P, Q, c, ws, dt, 2, bc3d=bc, metric=True)
    wt.step_rk4_curved(P, Q, c, ws, dt, 8, bc3d=bc, metric=True)
    assert abs(c.time - (t0 + 10 * dt)) < 1e-14
    Po, Qo = o.evolve_curved_td(kind, (A, d), t0, P0, Q0, dt, 10, bc=O.make_bc([2] * 6), use_metric=True)
    tol = 1e-12 if prec == 0 else 1e-5
    assert rel(P.double().cpu().numpy(), Po) < tol and rel(Q.double().cpu().numpy(), Qo) < tol
    # the device time the graph advanced is the one the coefficients hold (to the
    # round-off of adding dt step by step)
    c2 = wt.sample_background3d(g, kind, (A, d, t0 + 10 * dt))
    assert rel(c.get(), c2.get()) < 1e-13
    assert not ctx.nonfinite()


@pytest.mark.parametrize("kind", [4, 5])
def test_plane_wave_on_device(wt, ctx, kind):
    """The exact solution sin(k0 psi) on the periodic cube after t = 0.2 (n = 8, 4^3
    elements): error below 1e-5 (the oracle's own discretization error here is ~2e-6)."""
    import torch
    A, d, k0, t1 = 0.1, 1.0, 2 * np.pi, 0.2
    g = wt.Mesh.uniform_hex(ctx, 8, 4, periodic=True)
    c = wt.sample_background3d(g, kind, (A, d, 0.0))
    ws = wt.make_wave3d_workspace(g)
    x = g.get("coords").reshape(-1, 3)[:, 0]
    P0, Q0 = exact(kind, A, d, k0, 0.0, x)
    speed = 1.0 if kind == 4 else (1 + A) / (1 - A)
    nst = int(np.ceil(t1 / (0.2 * g.min_spacing() / speed)))
    P = torch.tensor(P0, dtype=torch.float64, device="cuda")
    Q = torch.tensor(Q0, dtype=torch.float64, device="cuda")
    wt.step_rk4_curved(P, Q, c, ws, t1 / nst, nst)
    Pe, _ = exact(kind, A, d, k0, t1, x)
    assert np.sqrt(np.mean((P.cpu().numpy() - Pe) ** 2)) < 1e-5
    # the same solve as a batch member (background re-sampled inside the batch graph)
    c2 = wt.sample_background3d(g, kind, (A, d, 0.0))
    ws2 = wt.make_wave3d_workspace(g)
    P2 = torch.tensor(P0, dtype=torch.float64, device="cuda")
    Q2 = torch.tensor(Q0, dtype=torch.float64, device="cuda")
    batch = wt.Batch(ctx)
    batch.add(P2, Q2, c2, ws2, t1 / nst)
    batch.step(nst)
    assert abs(c2.time - t1) < 1e-13
    assert np.sqrt(np.mean((P2.cpu().numpy() - Pe) ** 2)) < 1e-5
    batch.close()
