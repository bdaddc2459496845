"""Committed golden vectors (tests/golden/golden.npz, made by tests/golden/make_golden.py).

CPU: closed-form GLL known answers; the oracle reproduces every stored output
from the stored inputs; the library's host-side GLL operators equal the stored
ones bit for bit.  GPU: the library reproduces every stored output through the
C ABI (<= 1e-12 relative L2, energies <= 1e-11).
"""
import math
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "golden.npz")


@pytest.fixture(scope="module")
def G():
    return dict(np.load(GOLDEN))


def rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


# Gauss-Lobatto-Legendre nodes and weights on [-1, 1] in closed form (Abramowitz &
# Stegun 25.4.32), mapped to [0, 1]: x -> (1 + x)/2, w -> w/2.
KNOWN = {
    3: ([-1, 0, 1], [1 / 3, 4 / 3, 1 / 3]),
    4: ([-1, -1 / math.sqrt(5), 1 / math.sqrt(5), 1], [1 / 6, 5 / 6, 5 / 6, 1 / 6]),
    5: ([-1, -math.sqrt(3 / 7), 0, math.sqrt(3 / 7), 1], [1 / 10, 49 / 90, 32 / 45, 49 / 90, 1 / 10]),
}


@pytest.mark.parametrize("N", sorted(KNOWN))
def test_gll_known_answers(G, N):
    xs, ws = KNOWN[N]
    x = (1 + np.array(xs)) / 2
    w = np.array(ws) / 2
    assert np.max(np.abs(G[f"gll_N{N}_x"] - x)) < 4e-16
    assert np.max(np.abs(G[f"gll_N{N}_H"] - w)) < 4e-16
    # G differentiates polynomials of degree N-1 exactly
    D = G[f"gll_N{N}_G"]
    for k in range(N):
        assert np.max(np.abs(D @ x ** k - k * x ** max(k - 1, 0) * (k > 0))) < 1e-13


def test_gll_fixture_matches_oracle_and_library(G, O, wt):
    for N in range(2, 9):
        x, H, D = O.gll_ops(N)
        assert np.array_equal(x, G[f"gll_N{N}_x"]) and np.array_equal(H, G[f"gll_N{N}_H"])
        assert np.array_equal(D, G[f"gll_N{N}_G"])
        lx, lH, lD = wt.gll_operators(N)
        assert np.array_equal(np.asarray(lx), x) and np.array_equal(np.asarray(lH), H)
        assert np.array_equal(np.asarray(lD).reshape(N, N), D)


def test_oracle_reproduces_fixtures(G, O, wt):
    W = wt.workloads
    o = O.OracleMesh(4, (2, 2, 2), A=0.05, outer_tag=7)
    co = o.background(2, G["curved_warped_params"])
    Pd, Qd = o.rhs_curved(co, G["curved_warped_Phi"], G["curved_warped_Pi"], eps_ko=0.1,
                          bc=O.make_bc([2] * 6), use_metric=True)
    assert rel(Pd, G["curved_warped_Phidot"]) < 1e-13 and rel(Qd, G["curved_warped_Pidot"]) < 1e-13

    o = O.OracleMesh(5, (2, 3, 2), A=0.0, outer_tag=0)
    co = o.background(2, G["curved_affine_params"])
    d = G["curved_affine_bcdata"]
    bc = O.make_bc([1] * 6, gPhi=d[0], gPi=d[1], gDx=d[2], gDy=d[3], gDz=d[4])
    Pd, Qd = o.rhs_curved(co, G["curved_affine_Phi"], G["curved_affine_Pi"], eps_ko=0.0, bc=bc, use_metric=False)
    assert rel(Pd, G["curved_affine_Phidot"]) < 1e-13 and rel(Qd, G["curved_affine_Pidot"]) < 1e-13

    o = O.OracleMesh(6, 4, outer_tag=0)
    u0 = G["sipg_c1_u0"]
    assert rel(o.rhs_sipg(u0, np.zeros_like(u0), tau=20.0), G["sipg_c1_utt"]) < 1e-13
    u, v, E = o.evolve_sipg(u0, np.zeros_like(u0), float(G["sipg_c1_dt"][0]), 10, tau=20.0, eps_ko=0.1,
                            record_energy=True)
    assert rel(u, G["sipg_c1_u10"]) < 1e-13 and rel(v, G["sipg_c1_v10"]) < 1e-13
    assert np.max(np.abs(E / G["sipg_c1_energy"] - 1)) < 1e-12

    o = O.OracleMesh(5, 2, A=0.05, outer_tag=7)
    utt = o.rhs_strong(G["strong_warped_u"], G["strong_warped_ut"], R=1.0)
    assert rel(utt, G["strong_warped_utt"]) < 1e-13

    o = O.OracleMesh(8, 2, A=0.05, outer_tag=7)
    co = o.background(2, G["evolve_n8_params"])
    Phi = G["evolve_n8_Phi0"]
    P5, Q5, E = o.evolve_curved(co, Phi, np.zeros_like(Phi), float(G["evolve_n8_dt"][0]), 5,
                                bc=O.make_bc([2] * 6), use_metric=True, record_energy=True)
    assert rel(P5, G["evolve_n8_Phi5"]) < 1e-13 and rel(Q5, G["evolve_n8_Pi5"]) < 1e-13
    assert np.max(np.abs(E / G["evolve_n8_energy"] - 1)) < 1e-12
    # the stored inputs are the seeded workload generators' outputs
    x, y, z = o.coords()
    assert rel(W.gaussian_field(x, y, z, *W.pulses(3, 8)), Phi) < 1e-15


@pytest.mark.gpu
def test_library_reproduces_fixtures(G, wt, ctx):
    import torch

    def dev(a):
        return torch.tensor(np.asarray(a), dtype=torch.float64, device="cuda")

    def host(t):
        return t.double().cpu().numpy()

    m = wt.Mesh.uniform_hex(ctx, 4, (2, 2, 2), outer_tag=7, warp_A=0.05)
    c = wt.sample_background3d(m, wt.BG_ADM_PERTURBED, G["curved_warped_params"])
    ws = wt.make_wave3d_workspace(m)
    Pd, Qd = m.zeros(), m.zeros()
    wt.wave3d_curved_rhs(Pd, Qd, dev(G["curved_warped_Phi"]), dev(G["curved_warped_Pi"]), c, ws, eps_KO=0.1,
                         bc3d=wt.make_bc3d([2] * 6), metric=True)
    assert rel(host(Pd), G["curved_warped_Phidot"]) < 1e-12 and rel(host(Qd), G["curved_warped_Pidot"]) < 1e-12

    m = wt.Mesh.uniform_hex(ctx, 5, (2, 3, 2), outer_tag=0)
    c = wt.sample_background3d(m, wt.BG_ADM_PERTURBED, G["curved_affine_params"])
    ws = wt.make_wave3d_workspace(m)
    d = [dev(r) for r in G["curved_affine_bcdata"]]
    bc = wt.make_bc3d([1] * 6, gPhi=d[0], gPi=d[1], gDx=d[2], gDy=d[3], gDz=d[4])
    Pd, Qd = m.zeros(), m.zeros()
    wt.wave3d_curved_rhs(Pd, Qd, dev(G["curved_affine_Phi"]), dev(G["curved_affine_Pi"]), c, ws, eps_KO=0.0,
                         bc3d=bc, metric=False)
    assert rel(host(Pd), G["curved_affine_Phidot"]) < 1e-12 and rel(host(Qd), G["curved_affine_Pidot"]) < 1e-12

    m = wt.Mesh.uniform_hex(ctx, 6, 4, outer_tag=0)
    ws = wt.make_wave3d_workspace(m)
    u0 = dev(G["sipg_c1_u0"])
    utt = m.zeros()
    wt.rhs_wave3d(utt, u0, m.zeros(), [0] * 6, ws, tau=20.0)
    assert rel(host(utt), G["sipg_c1_utt"]) < 1e-12
    u, v = u0.clone(), m.zeros()
    E0 = wt.energy_sipg(u, v, ws, 20.0)
    wt.step_rk4_sipg(u, v, ws, float(G["sipg_c1_dt"][0]), 10, tau=20.0, eps_KO=0.1)
    assert rel(host(u), G["sipg_c1_u10"]) < 1e-12 and rel(host(v), G["sipg_c1_v10"]) < 1e-12
    assert abs(E0 / G["sipg_c1_energy"][0] - 1) < 1e-11
    assert abs(wt.energy_sipg(u, v, ws, 20.0) / G["sipg_c1_energy"][-1] - 1) < 1e-11

    m = wt.Mesh.uniform_hex(ctx, 5, 2, outer_tag=7, warp_A=0.05)
    ws = wt.make_wave3d_workspace(m)
    utt = m.zeros()
    wt.wave_strong_rhs_mesh(utt, dev(G["strong_warped_u"]), dev(G["strong_warped_ut"]), ws, sommerfeld_R=1.0)
    assert rel(host(utt), G["strong_warped_utt"]) < 1e-12

    m = wt.Mesh.uniform_hex(ctx, 8, 2, outer_tag=7, warp_A=0.05)
    c = wt.sample_background3d(m, wt.BG_ADM_PERTURBED, G["evolve_n8_params"])
    ws = wt.make_wave3d_workspace(m)
    P, Q = dev(G["evolve_n8_Phi0"]), m.zeros()
    wt.step_rk4_curved(P, Q, c, ws, float(G["evolve_n8_dt"][0]), 5, bc3d=wt.make_bc3d([2] * 6), metric=True)
    assert rel(host(P), G["evolve_n8_Phi5"]) < 1e-12 and rel(host(Q), G["evolve_n8_Pi5"]) < 1e-12
    E = wt.wave3d_energy(P, Q, c, ws, metric=True)
    assert abs(E / G["evolve_n8_energy"][-1] - 1) < 1e-11
