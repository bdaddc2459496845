"""GPU: the lapse-weighted energy (wt_energy_lapse).

The reference's wave3d_energy is exactly conserved only for alpha = 1
(src/wave3d_curved.jl:263-266).  For a static background with zero shift the
split-form semi-discretisation conserves the reference energy's integrand times
the lapse, E_alpha = sum 1/2 [(alpha/sqrtg) Pi^2 + alpha sqrtg gu^{ij} dPhi_i dPhi_j] Hd
(the CPU oracle's property test shows dE_alpha/dt = 0 to round-off).  Here the
device reduction matches the oracle's, and over RK4 steps E_alpha does not
grow (the classic RK4 only dissipates a little) while the reference energy
grows by a visible amount.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _no_shift(wt, seed, scale):
    p = list(wt.workloads.adm_params(seed, scale))
    p[1] = 0.0   # beta = 0
    return p


@pytest.mark.parametrize("N,M,periodic", [(6, 3, True), (8, 2, False), (5, (2, 3, 2), True)])
def test_energy_lapse_matches_oracle(wt, ctx, O, N, M, periodic):
    import torch
    g = wt.Mesh.uniform_hex(ctx, N, M, periodic=periodic, outer_tag=0 if periodic else 7, warp_A=0.05)
    o = O.OracleMesh(N, M, A=0.05, periodic=periodic, outer_tag=0 if periodic else 7)
    p = wt.workloads.adm_params(4, 1.5)
    cg, co = wt.sample_background3d(g, wt.BG_ADM_PERTURBED, p), o.background(2, p)
    ws = wt.make_wave3d_workspace(g)
    x, y, z = o.coords()
    Phi = wt.workloads.gaussian_field(x, y, z, *wt.workloads.pulses(4, 2))
    Pi = np.cos(2 * np.pi * (x + y)) * Phi
    Pg, Qg = torch.tensor(Phi, device="cuda"), torch.tensor(Pi, device="cuda")
    Eg = wt.wave3d_energy(Pg, Qg, cg, ws, metric=True, lapse=True)
    Eo = o.energy(co, Phi, Pi, use_metric=True, lapse=True)
    assert abs(Eg - Eo) <= 1e-12 * abs(Eo)
    # the reference energy is a different number for alpha != 1
    assert abs(wt.wave3d_energy(Pg, Qg, cg, ws, metric=True) - Eo) > 1e-6 * abs(Eo)


@pytest.mark.parametrize("prec", [0, 1])
def test_energy_lapse_does_not_grow(wt, ctx, prec):
    """Periodic warped mesh, static ADM background with zero shift and alpha != 1: 40 RK4
    steps (FP64, and the compensated FP32 form)."""
    N, M = 6, 3
    g = wt.Mesh.uniform_hex(ctx, N, M, periodic=True, warp_A=0.05, precision=prec)
    p = _no_shift(wt, 7, 2.0)
    c = wt.sample_background3d(g, wt.BG_ADM_PERTURBED, p)
    ws = wt.make_wave3d_workspace(g)
    P, Q = g.zeros(), g.zeros()
    wt.initial_state(ws, wt.IC_GAUSSIANS, wt.gaussian_params(*wt.workloads.pulses(3, 2)), P, Q)
    dt = 0.2 * g.min_spacing() / wt.workloads.max_speed(p)
    Ea0 = wt.wave3d_energy(P, Q, c, ws, metric=True, lapse=True)
    E0 = wt.wave3d_energy(P, Q, c, ws, metric=True)
    wt.step_rk4_curved(P, Q, c, ws, dt, 40, metric=True)
    Ea1 = wt.wave3d_energy(P, Q, c, ws, metric=True, lapse=True)
    E1 = wt.wave3d_energy(P, Q, c, ws, metric=True)
    up = 1e-9 if prec == 0 else 1e-6   # FP32: the energy of the rounded (high-part) state
    assert Ea1 <= Ea0 * (1 + up) and Ea1 >= Ea0 * (1 - 1e-6)
    assert E1 / E0 - 1 > 1e-3
    assert not ctx.nonfinite()
