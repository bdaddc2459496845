"""GPU parity of the scalar wave on a prescribed 4-metric (wt_curved4_background,
wt_rhs_curved4 = eval_curved_background!, wave_curved_rhs_mesh! and
wave_curved_rhs_conservative_mesh!) against the CPU Float64 oracle: <= 1e-12
relative L2 (FP64), <= 1e-5 (FP32)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


@pytest.mark.parametrize("N,M,periodic,prec", [(4, 2, True, 0), (6, 2, False, 0), (8, 2, True, 0),
                                              (5, 3, True, 1)])
def test_curved4_matches_oracle(wt, ctx, O, N, M, periodic, prec):
    import torch
    dtype = torch.float64 if prec == 0 else torch.float32
    tol = 1e-12 if prec == 0 else 1e-5
    g = wt.Mesh.uniform_hex(ctx, N, M, 0.0, 1.0, periodic=periodic, precision=prec)
    o = O.OracleMesh(N, M, periodic=periodic)
    h = 1.0 / M
    ws = wt.make_wave3d_workspace(g)
    ginv = torch.zeros(10 * g.nn, dtype=dtype, device="cuda")
    gam = torch.zeros(4 * g.nn, dtype=dtype, device="cuda")
    wt.eval_curved_background(ginv, gam, g, wt.CURVED4_GAUGE_WAVE, (0.1, 1.0), 0.13)
    go, Go = o.curved4_background(1, (0.1, 1.0), 0.13)
    assert rel(ginv.double().cpu().numpy(), go) < (1e-14 if prec == 0 else 1e-7)
    assert np.max(np.abs(gam.double().cpu().numpy())) == 0.0
    rng = np.random.default_rng(N * 10 + prec)
    x, y, z = o.coords()
    phi = np.sin(2 * np.pi * x) * np.cos(2 * np.pi * y) * np.sin(2 * np.pi * z) + 0.1 * rng.standard_normal(o.nn)
    phid = 0.5 * rng.standard_normal(o.nn)
    out = g.zeros()
    for cons in (False, True):
        wt.wave_curved_rhs_mesh(out, torch.tensor(phi, dtype=dtype, device="cuda"),
                                torch.tensor(phid, dtype=dtype, device="cuda"), ginv, gam, ws, h, conservative=cons)
        ref = o.rhs_curved4(phi, phid, go, Go, h, conservative=cons)
        assert rel(out.double().cpu().numpy(), ref) < tol, cons


def test_curved4_minkowski_equals_flat_conservative_laplacian(wt, ctx):
    import torch
    g = wt.Mesh.uniform_hex(ctx, 6, 3, 0.0, 1.0, periodic=True)
    ws = wt.make_wave3d_workspace(g)
    ginv = torch.zeros(10 * g.nn, dtype=torch.float64, device="cuda")
    gam = torch.zeros(4 * g.nn, dtype=torch.float64, device="cuda")
    wt.eval_curved_background(ginv, gam, g, wt.CURVED4_MINKOWSKI)
    phi = torch.randn(g.nn, dtype=torch.float64, device="cuda")
    a, b = g.zeros(), g.zeros()
    wt.wave_curved_rhs_mesh(a, phi, torch.randn_like(phi), ginv, gam, ws, 1.0 / 3, conservative=True)
    wt.wave_lap_strong_conservative_mesh(b, phi, 1.0 / 3, ws)
    assert rel(a.cpu().numpy(), b.cpu().numpy()) < 1e-12


def test_curved4_rejects_bad_arguments(wt, ctx):
    import torch
    g = wt.Mesh.uniform_hex(ctx, 4, 2, 0.0, 1.0, periodic=True)
    ws = wt.make_wave3d_workspace(g)
    ginv = torch.zeros(10 * g.nn, dtype=torch.float64, device="cuda")
    gam = torch.zeros(4 * g.nn, dtype=torch.float64, device="cuda")
    with pytest.raises(wt.WaveToyError):
        wt.eval_curved_background(ginv, gam, g, 7)
    with pytest.raises(wt.WaveToyError):
        wt.eval_curved_background(ginv, gam, g, wt.CURVED4_GAUGE_WAVE, (1.5, 1.0))
    with pytest.raises(wt.WaveToyError):
        wt.wave_curved_rhs_mesh(g.zeros(), g.zeros(), g.zeros(), ginv, gam, ws, 0.0)
    w = wt.Mesh.uniform_hex(ctx, 4, 2, 0.0, 1.0, warp_A=0.05)
    with pytest.raises(wt.WaveToyError):
        wt.wave_curved_rhs_mesh(w.zeros(), w.zeros(), w.zeros(), torch.zeros(10 * w.nn, dtype=torch.float64,
                                device="cuda"), torch.zeros(4 * w.nn, dtype=torch.float64, device="cuda"),
                                wt.make_wave3d_workspace(w), 0.5)
