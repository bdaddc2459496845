"""GPU: evolve3d in one call (wt_evolve3d).

The call equals the same solve built and stepped through the individual
entry points (mesh, background, workspace, initial state, RK4 steps of the
sampling schedule with the shortened last step, energies at the samples), bit
for bit.  The time-sampling rules follow the reference's loop
(src/evolve.jl:1311-1318).  With the eigenmode (an exact solution of the periodic
Minkowski problem) l2_err is the distance to it, 0 at t0 and small after, and
the energy is conserved.  Dissipation limits dt by 1.4 / (eps_KO mu).  The call
leaves no device memory behind.
"""
import gc
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _adm_desc(wt, prec=0, **kw):
    p = wt.workloads.adm_params(4)
    args = dict(N=8, M=2, T=prec, warp_A=0.05, background=wt.BG_ADM_PERTURBED, bg_params=p,
                ic=wt.IC_GAUSSIANS, ic_params=wt.gaussian_params(*wt.workloads.pulses(4, 2)),
                bc3d=wt.make_bc3d([wt.BC_SOMMERFELD] * 6), t1=0.05, Nt=4, cfl=0.2,
                max_speed=wt.workloads.max_speed(p))
    args.update(kw)
    return wt.solve_desc(**args), p


@pytest.mark.parametrize("prec", [0, 1])
def test_evolve3d_equals_the_manual_solve(wt, ctx, prec):
    import torch
    gc.collect()
    base = ctx.memory()[0]
    d, p = _adm_desc(wt, prec)
    r = wt.evolve3d(ctx, d)
    gc.collect()
    assert ctx.memory()[0] == base                       # everything released
    # the same solve through the individual entry points
    g = wt.Mesh.uniform_hex(ctx, 8, 2, outer_tag=7, warp_A=0.05, precision=prec)
    c = wt.sample_background3d(g, wt.BG_ADM_PERTURBED, p)
    ws = wt.make_wave3d_workspace(g)
    P, Q = g.zeros(), g.zeros()
    wt.initial_state(ws, wt.IC_GAUSSIANS, wt.gaussian_params(*wt.workloads.pulses(4, 2)), P, Q)
    dt = r["dt"]
    ref_dt = 0.2 * g.min_spacing() / wt.workloads.max_speed(p)
    assert dt == (ref_dt if prec == 0 else float(np.float32(np.float32(0.2) * np.float32(g.min_spacing())
                                                            / np.float32(wt.workloads.max_speed(p)))))
    steps, last, ts = wt.solve_schedule(0.0, 0.05, 4, dt, prec)
    assert r["steps"] == steps.sum() and np.array_equal(r["ts_actual"], ts)
    assert ts[-1] == (0.05 if prec == 0 else float(np.float32(0.05)))   # t1 in the time type
    bc = wt.make_bc3d([wt.BC_SOMMERFELD] * 6)
    E = []
    final = max(n for n in range(4) if steps[n] > 0)
    for n in range(4):
        k = int(steps[n]) - (1 if n == final and last != dt else 0)
        if k:
            wt.step_rk4_curved(P, Q, c, ws, dt, k, bc3d=bc, metric=True)
        if n == final and last != dt:
            wt.step_rk4_curved(P, Q, c, ws, last, 1, bc3d=bc, metric=True)
        E.append(wt.wave3d_energy(P, Q, c, ws, metric=True))
    assert np.array_equal(r["Phi_final"], P.cpu().numpy()) and np.array_equal(r["Pi_final"], Q.cpu().numpy())
    assert np.array_equal(r["energy"], np.array(E))
    # the 1-D slice at the mid-plane: the rule of the reference's _build_slice_3d on the mesh
    # coordinates, and at the last sample the final state's values there
    xyz = g.get("coords").reshape(-1, 3)
    atol = float(np.sqrt(np.finfo(np.float64 if prec == 0 else np.float32).eps))
    nodes, xs = wt.slice_select(xyz, 0.5, 0.5, atol)
    assert len(nodes) > 0 and np.array_equal(r["slice_nodes"], nodes) and np.array_equal(r["xs_line"], xs)
    assert r["Phis"].shape == (len(nodes), 4)
    assert np.array_equal(r["Phis"][:, -1], r["Phi_final"][nodes].astype(np.float64))
    assert np.array_equal(r["Pis"][:, -1], r["Pi_final"][nodes].astype(np.float64))


def test_evolve3d_exact_solution_and_energy(wt, ctx):
    k = 2 * math.pi
    d = wt.solve_desc(N=8, M=4, periodic=True, background=wt.BG_MINKOWSKI, ic=wt.IC_EIGENMODE_CARTESIAN,
                      ic_params=[1.0, k, k, k, math.sqrt(3) * k, 0.0, 1.0], ic_exact=True, t1=0.2, Nt=5,
                      cfl=0.2, metric=False)
    r = wt.evolve3d(ctx, d)
    assert r["l2_err"][0] <= 1e-15
    assert 0 < r["l2_err"][-1] < 1e-4                   # n = 8, 4 elements per wavelength
    assert np.all(np.abs(r["energy"] / r["energy"][0] - 1) < 1e-6)
    assert r["ts_actual"][-1] == 0.2 and r["mu"] == 0


def test_evolve3d_dissipation_limits_dt_and_patch_meshes_run(wt, ctx):
    d, p = _adm_desc(wt, 0, N=6, M=3, eps_KO=40.0, cfl=10.0, Nt=3, t1=0.01)
    r = wt.evolve3d(ctx, d)
    assert r["mu"] > 0 and r["dt"] == pytest.approx(1.4 / (40.0 * r["mu"]), rel=1e-15)
    assert np.all(np.isfinite(r["Phi_final"]))
    q = wt.solve_desc(N=5, M=2, mesh_kind=wt.MESH_CUBED_CUBE, patch_params=(0.3,),
                      background=wt.BG_ADM_PERTURBED, bg_params=wt.workloads.adm_params(3),
                      ic=wt.IC_GAUSSIANS, ic_params=wt.gaussian_params(*wt.workloads.pulses(3, 1)),
                      bc3d=wt.make_bc3d([wt.BC_SOMMERFELD] * 6), t1=0.02, Nt=3, cfl=0.2, max_speed=2.0)
    r = wt.evolve3d(ctx, q)
    assert r["Phi_final"].size == 7 * 8 * 125 and np.all(np.isfinite(r["energy"]))
    with pytest.raises(wt.WaveToyError) as ei:
        wt.evolve3d(ctx, wt.solve_desc(Nt=0))
    assert ei.value.code == -1
