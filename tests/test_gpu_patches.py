"""GPU parity on multi-patch meshes and turned elements (face orientation != 0).

The library's meshes (wt_mesh_create_patches; wt_mesh_create_arrays with the
orientation inferred from the coordinates) against the oracle built from the
same arrays: the curvilinear RHS with Sommerfeld outer faces, the radial
shell's excised inner sphere, Kreiss-Oliger (applied by apply_D! passes where
the elements form no straight lines) and RK4 -- through the generic kernels
(n = 4, 5), the n = 8 FP64 tensor-core kernels and the FP32 forms.  Bars:
<= 1e-12 relative L2 (FP64; 5e-12 for one n = 8 tensor-core RHS), <= 5e-5 (FP32)."""
import numpy as np
import pytest

from test_patch_meshes import KINDS, oracle_from, turned_mesh

pytestmark = pytest.mark.gpu


def rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def host(x):
    return x.detach().double().cpu().numpy()


def smooth(x, y, z, seed):
    rng = np.random.default_rng(seed)
    k = rng.uniform(1.0, 3.0, 3)
    return np.sin(k[0] * x + 0.3) * np.cos(k[1] * y - 0.2) * np.sin(k[2] * z + 0.5) + 0.2 * np.cos(x + y - z)


@pytest.mark.parametrize("kind,M,p", KINDS)
@pytest.mark.parametrize("N,prec,form", [(4, 0, None), (8, 0, None), (8, 1, 0), (8, 1, 1)])
def test_patch_rhs_matches_oracle(wt, ctx, O, kind, M, p, N, prec, form):
    import torch
    g = wt.Mesh.patches(ctx, kind, N, M, p, precision=prec)
    if form is not None:
        g.set_fp32_form(form)
    a = wt.patch_mesh_arrays(kind, N, M, p)
    assert np.array_equal(g.get("orientation"), a["orientation"])
    o = oracle_from(O, N, a)
    prm = wt.workloads.adm_params(3)
    cg, co = wt.sample_background3d(g, wt.BG_ADM_PERTURBED, prm), o.background(2, prm)
    ws = wt.make_wave3d_workspace(g)
    x, y, z = o.coords()
    Phi, Pi = smooth(x, y, z, 1), 0.3 * smooth(x, y, z, 2)
    dt_ = torch.float64 if prec == 0 else torch.float32
    dev = lambda v: torch.tensor(v, dtype=dt_, device="cuda")
    for eps in (0.0, 0.1):
        Pd, Qd = g.zeros(), g.zeros()
        wt.wave3d_curved_rhs(Pd, Qd, dev(Phi), dev(Pi), cg, ws, eps_KO=eps,
                             bc3d=wt.make_bc3d([2] * 6, excision_tag=8), metric=True)
        Po, Qo = o.rhs_curved(co, Phi, Pi, eps_ko=eps, bc=O.make_bc([2] * 6, excision_tag=8), use_metric=True)
        # FP32: input rounding (6e-8) amplified by the second derivatives of Pi-dot
        # on these meshes reaches ~2e-5 of the RHS norm (orientation errors would be O(1))
        tol = (5e-12 if N == 8 else 1e-12) if prec == 0 else 5e-5
        assert rel(host(Pd), Po) < tol and rel(host(Qd), Qo) < tol, (eps, rel(host(Pd), Po), rel(host(Qd), Qo))
    assert not ctx.nonfinite()


@pytest.mark.parametrize("kind,M,p", KINDS)
def test_patch_free_stream_and_rk4(wt, ctx, O, kind, M, p):
    """Constant data stays constant on the device (n = 8, FP64); RK4 with
    Kreiss-Oliger over 6 steps matches the oracle (n = 5)."""
    import torch
    g = wt.Mesh.patches(ctx, kind, 8, M, p)
    c0 = wt.sample_background3d(g, wt.BG_MINKOWSKI)
    ws = wt.make_wave3d_workspace(g)
    Pd, Qd = g.zeros(), g.zeros()
    wt.wave3d_curved_rhs(Pd, Qd, torch.full((g.nn,), 2.5, dtype=torch.float64, device="cuda"), g.zeros(), c0, ws,
                         eps_KO=0.0, bc3d=wt.make_bc3d([2] * 6, excision_tag=8), metric=True)
    assert host(Pd).__abs__().max() <= 1e-9 and host(Qd).__abs__().max() <= 1e-9
    N = 5
    g = wt.Mesh.patches(ctx, kind, N, M, p)
    o = oracle_from(O, N, wt.patch_mesh_arrays(kind, N, M, p))
    prm = wt.workloads.adm_params(4)
    cg, co = wt.sample_background3d(g, wt.BG_ADM_PERTURBED, prm), o.background(2, prm)
    ws = wt.make_wave3d_workspace(g)
    x, y, z = o.coords()
    Phi, Pi = smooth(x, y, z, 3), np.zeros(o.nn)
    dt = 0.2 * o.min_spacing() / wt.workloads.max_speed(prm)
    Pg = torch.tensor(Phi, dtype=torch.float64, device="cuda")
    Qg = torch.tensor(Pi, dtype=torch.float64, device="cuda")
    wt.step_rk4_curved(Pg, Qg, cg, ws, dt, 6, eps_KO=0.1, bc3d=wt.make_bc3d([2] * 6, excision_tag=8), metric=True)
    Po, Qo = o.evolve_curved(co, Phi, Pi, dt, 6, eps_ko=0.1, bc=O.make_bc([2] * 6, excision_tag=8), use_metric=True)
    assert rel(host(Pg), Po) < 1e-12 and rel(host(Qg), Qo) < 1e-12
    assert not ctx.nonfinite()


@pytest.mark.parametrize("N", [5, 8])
def test_turned_elements_infer_orientation(wt, ctx, O, N):
    """A warped mesh with randomly turned elements through wt_mesh_create_arrays: the
    library infers every orientation code from the coordinates, and its RHS and RK4
    states match the oracle's on the same arrays (every code through the SAT reads
    of the generic and the n = 8 kernels)."""
    import torch
    base = O.OracleMesh(N, 3, A=0.05, outer_tag=7)
    arr, _ = turned_mesh(O, base, N, 11)
    g = wt.Mesh.from_arrays(ctx, N, arr["coords"], arr["jac"], arr["neighbour"], arr["neighbour_face"],
                            np.zeros_like(arr["orientation"]), arr["bdry"])
    assert np.array_equal(g.get("orientation"), arr["orientation"])
    assert set(arr["orientation"][arr["neighbour"] > 0]) == set(range(8))
    o = oracle_from(O, N, arr)
    prm = wt.workloads.adm_params(6)
    cg, co = wt.sample_background3d(g, wt.BG_ADM_PERTURBED, prm), o.background(2, prm)
    ws = wt.make_wave3d_workspace(g)
    x, y, z = o.coords()
    Phi, Pi = smooth(x, y, z, 5), 0.2 * smooth(x, y, z, 6)
    Pd, Qd = g.zeros(), g.zeros()
    dev = lambda v: torch.tensor(v, dtype=torch.float64, device="cuda")
    bc_g, bc_o = wt.make_bc3d([2] * 6), O.make_bc([2] * 6)
    wt.wave3d_curved_rhs(Pd, Qd, dev(Phi), dev(Pi), cg, ws, eps_KO=0.1, bc3d=bc_g, metric=True)
    Po, Qo = o.rhs_curved(co, Phi, Pi, eps_ko=0.1, bc=bc_o, use_metric=True)
    tol = 5e-12 if N == 8 else 1e-12
    assert rel(host(Pd), Po) < tol and rel(host(Qd), Qo) < tol
    dt = 0.2 * o.min_spacing() / wt.workloads.max_speed(prm)
    Pg, Qg = dev(Phi), dev(Pi)
    wt.step_rk4_curved(Pg, Qg, cg, ws, dt, 4, bc3d=bc_g, metric=True)
    Pe, Qe = o.evolve_curved(co, Phi, Pi, dt, 4, bc=bc_o, use_metric=True)
    assert rel(host(Pg), Pe) < 1e-12 and rel(host(Qg), Qe) < 1e-12


def test_patch_mesh_errors(wt, ctx):
    with pytest.raises(wt.WaveToyError):
        wt.Mesh.patches(ctx, 9, 4, 2, (0.3,))
    with pytest.raises(wt.WaveToyError):
        wt.Mesh.patches(ctx, wt.MESH_CUBED_CUBE, 4, 2, (1.5,))
    with pytest.raises(wt.WaveToyError):
        wt.Mesh.patches(ctx, wt.MESH_RADIAL_SHELL, 4, 2, (1.0, 0.5))
    # faces that do not coincide under any orientation, nor up to one shift (periodic faces)
    a = wt.patch_mesh_arrays(wt.MESH_CUBED_CUBE, 4, 1, (0.3,))
    c = a["coords"].copy()
    c[: 3 * 64] *= 1.01
    with pytest.raises(wt.WaveToyError):
        wt.Mesh.from_arrays(ctx, 4, c, a["jac"], a["neighbour"], a["neighbour_face"], a["orientation"], a["bdry"])


@pytest.mark.parametrize("kind,M,p", KINDS)
@pytest.mark.parametrize("N", [4, 8])
def test_patch_compensated_fp32_rk4(wt, ctx, O, kind, M, p, N):
    """The default FP32 form (compensated: Phi carried as high + low part, FP64 gradient
    of Phi) on multi-patch meshes, through the generic (n = 4) and the n = 8 kernels with
    every face orientation the patches have: 30 RK4 steps from an FP64 state loaded by
    wt_state_set_f64, against the oracle, <= 1e-5."""
    import torch
    g = wt.Mesh.patches(ctx, kind, N, M, p, precision=1)
    o = oracle_from(O, N, wt.patch_mesh_arrays(kind, N, M, p))
    prm = wt.workloads.adm_params(8)
    cg, co = wt.sample_background3d(g, wt.BG_ADM_PERTURBED, prm), o.background(2, prm)
    ws = wt.make_wave3d_workspace(g)
    x, y, z = o.coords()
    Phi, Pi = smooth(x, y, z, 7), 0.2 * smooth(x, y, z, 8)
    P, Q = g.zeros(), g.zeros()
    d64 = lambda v: torch.tensor(v, dtype=torch.float64, device="cuda")
    wt.state_from_f64(ws, d64(Phi), d64(Pi), P, Q)
    dt = 0.2 * o.min_spacing() / wt.workloads.max_speed(prm)
    bc_g, bc_o = wt.make_bc3d([2] * 6, excision_tag=8), O.make_bc([2] * 6, excision_tag=8)
    wt.step_rk4_curved(P, Q, cg, ws, dt, 30, bc3d=bc_g, metric=True)
    Po, Qo = o.evolve_curved(co, Phi, Pi, dt, 30, bc=bc_o, use_metric=True)
    err = rel(np.concatenate([host(P), host(Q)]), np.concatenate([Po, Qo]))
    assert err <= 1e-5, err
    assert not ctx.nonfinite()
