"""GPU: one solve split into z-slabs (wt_mesh_create_slab, wt_rk4_stage_curved,
wt_halo_copy; or wt_rk4_stage_curved_layers and wt_halo_face_copy; slabs.py)
advances its owned element layers exactly as the
undivided mesh does -- bit for bit, since every element's arithmetic depends
only on its own data and its neighbours' face traces, which the halo exchange
supplies -- through the n = 8 FP64 tensor-core kernels, the generic kernels, the
FP32 CUDA-core and split-BF16 forms, a periodic ring of slabs and a time-dependent background
re-sampled at every stage.  The slabs share one device here (in-process
exchange); between GPUs the same messages go through torch.distributed."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = [  # N, M, slabs, periodic, precision, fp32 form, background
    (8, (3, 2, 6), 2, False, 0, None, 2),
    (8, (2, 3, 7), 3, True, 0, None, 2),
    (5, (3, 3, 5), 2, False, 0, None, 2),
    (8, (2, 2, 6), 3, False, 1, 0, 2),
    (8, (2, 2, 5), 2, False, 1, 1, 2),     # split-BF16 form: 544-word flux blocks
    (6, (2, 2, 6), 2, True, 0, None, 4),
    (8, (2, 2, 6), 3, False, 1, 3, 2),     # compensated FP32 form: the halo also carries Phi's small part
    (6, (2, 3, 6), 2, True, 1, 3, 2),      # compensated, generic kernels, periodic ring
    (6, (2, 2, 4), 3, False, 0, None, 2),  # slabs of 2, 1 and 1 layers: a one-layer slab between two cuts
]


@pytest.mark.parametrize("halo", ["layers", "faces"])
@pytest.mark.parametrize("N,M,nslabs,periodic,prec,form,bg", CASES)
def test_slab_solve_equals_whole_mesh(wt, ctx, N, M, nslabs, periodic, prec, form, bg, halo):
    """halo "layers": every slab layer computed, whole ghost layers exchanged after the first
    stage half (step, LocalHalo); "faces": owned layers only, the shared face planes exchanged
    while the interior layers' first half runs (step_faces, LocalFaceHalo)."""
    import torch
    S = wt.slabs
    kw = dict(warp_A=0.05, periodic=periodic, outer_tag=0 if periodic else 7, precision=prec)
    prm = wt.workloads.adm_params(5) if bg == 2 else (0.1, 1.0, 0.05)
    speed = wt.workloads.max_speed(prm) if bg == 2 else 1.0
    ic = wt.gaussian_params(*wt.workloads.pulses(5, 2))
    bc = wt.make_bc3d([wt.BC_SOMMERFELD] * 6)
    whole = wt.Mesh.uniform_hex(ctx, N, M, **kw)
    if form is not None:
        whole.set_fp32_form(form)
    coef = wt.sample_background3d(whole, bg, prm)
    ws = wt.make_wave3d_workspace(whole)
    P, Q = whole.zeros(), whole.zeros()
    wt.initial_data(whole, wt.IC_GAUSSIANS, ic, P)
    dt = 0.2 * whole.min_spacing() / speed
    nsteps = 5
    wt.step_rk4_curved(P, Q, coef, ws, dt, nsteps, bc3d=bc, metric=True)

    slabs = [S.Slab(ctx, r, N, M, **kw, bg_kind=bg, bg_params=prm, fp32_form=form)
             for r in S.partition(M[2], nslabs, periodic)]
    for s in slabs:
        wt.initial_data(s.mesh, wt.IC_GAUSSIANS, ic, s.Phi)
    assert min(s.mesh.min_spacing() for s in slabs) == whole.min_spacing()
    if halo == "layers":
        S.step(slabs, S.LocalHalo(slabs), dt, nsteps, bc)
    else:
        S.step_faces(slabs, S.LocalFaceHalo(slabs), dt, nsteps, bc)
    Ps = torch.cat([s.owned(s.Phi) for s in slabs])
    Qs = torch.cat([s.owned(s.Pi) for s in slabs])
    assert torch.isfinite(Ps).all() and float(P.abs().max()) > 0
    assert torch.equal(Ps, P) and torch.equal(Qs, Q), (float((Ps - P).abs().max()), float((Qs - Q).abs().max()))
    if bg == 4:
        assert all(abs(s.coef.time - coef.time) < 1e-15 for s in slabs)
    for s in slabs:
        s.close()
    assert not ctx.nonfinite()


def test_stage_halves_equal_fused_step(wt, ctx):
    """Parts 1 and 2 of stages 0..3 called one by one are one wt_step_rk4_curved step."""
    import torch
    g = wt.Mesh.uniform_hex(ctx, 8, (2, 2, 3), warp_A=0.05, outer_tag=7)
    prm = wt.workloads.adm_params(2)
    c = wt.sample_background3d(g, wt.BG_ADM_PERTURBED, prm)
    ws1, ws2 = wt.make_wave3d_workspace(g), wt.make_wave3d_workspace(g)
    P1 = g.zeros()
    wt.initial_data(g, wt.IC_GAUSSIANS, wt.gaussian_params(*wt.workloads.pulses(2, 2)), P1)
    Q1 = 0.3 * P1
    P2, Q2 = P1.clone(), Q1.clone()
    bc = wt.make_bc3d([wt.BC_SOMMERFELD] * 6)
    dt = 1e-3
    wt.step_rk4_curved(P1, Q1, c, ws1, dt, 2, bc3d=bc, metric=True)
    for _ in range(2):
        for st in range(4):
            for part in (1, 2):
                wt.rk4_stage_curved(P2, Q2, c, ws2, dt, st, part, bc3d=bc, metric=True)
    assert torch.equal(P1, P2) and torch.equal(Q1, Q2)


def test_slab_errors(wt, ctx):
    with pytest.raises(wt.WaveToyError):          # layers outside a non-periodic mesh
        wt.Mesh.slab(ctx, 6, 3, 2, 2)
    with pytest.raises(wt.WaveToyError):
        wt.Mesh.slab(ctx, 6, 3, 0, 4, periodic=True)
    g = wt.Mesh.slab(ctx, 6, (2, 2, 5), -1, 3, periodic=True)
    assert g.Ne == 12
    ws = wt.make_wave3d_workspace(g)
    with pytest.raises(wt.WaveToyError):          # nothing to size before a stage has run
        wt.halo_size(ws)
    c = wt.sample_background3d(g, wt.BG_MINKOWSKI)
    P, Q = g.zeros(), g.zeros()
    with pytest.raises(wt.WaveToyError):
        wt.rk4_stage_curved(P, Q, c, ws, 1e-3, 4, 1, metric=True)
    wt.rk4_stage_curved(P, Q, c, ws, 1e-3, 0, 1, metric=True)
    n = wt.halo_size(ws)
    assert n == 4 * 6 ** 3 * 4                    # Phi + three flux components of 4 elements
    import torch
    buf = torch.empty(n, dtype=torch.float64, device="cuda")
    with pytest.raises(wt.WaveToyError):
        wt.halo_copy(ws, P, 0, 3, buf, True)      # the slab has layers 0..2
    wt.halo_copy(ws, P, 0, 2, buf, True)


# cubic elements: mu (the KO normalisation) is estimated along axis 1, so elements
# much thinner along z than along x would make mu^-5 D_z^6 too stiff for the step
@pytest.mark.parametrize("N,M,nslabs,periodic,prec", [(5, (12, 12, 12), 2, False, 0), (8, (12, 12, 12), 2, False, 0),
                                                      (6, (18, 18, 18), 3, True, 0), (8, (12, 12, 12), 2, False, 1)])
def test_dissipative_slab_solve_equals_whole_mesh(wt, ctx, N, M, nslabs, periodic, prec):
    """Kreiss-Oliger dissipation on slabs: six ghost layers per cut (its z passes reach
    six elements), whole stages on each slab and a state halo after every stage, the
    whole mesh's mu imposed on every slab -- the owned layers match the undivided
    solve to round-off (<= 1e-13 of the field's maximum in FP64; <= 1e-6 for the
    FP32 form, whose Kahan compensation of the RK4 sums is also kept on the ghost
    layers that the state halo overwrites)."""
    import torch
    S = wt.slabs
    kw = dict(warp_A=0.05, periodic=periodic, outer_tag=0 if periodic else 7, precision=prec)
    prm = wt.workloads.adm_params(7)
    ic = wt.gaussian_params(*wt.workloads.pulses(7, 2))
    bc = wt.make_bc3d([wt.BC_SOMMERFELD] * 6)
    whole = wt.Mesh.uniform_hex(ctx, N, M, **kw)
    coef = wt.sample_background3d(whole, wt.BG_ADM_PERTURBED, prm)
    ws = wt.make_wave3d_workspace(whole)
    P, Q = whole.zeros(), whole.zeros()
    wt.initial_data(whole, wt.IC_GAUSSIANS, ic, P)
    dt = 0.2 * whole.min_spacing() / wt.workloads.max_speed(prm)
    nsteps, eps = 4, 0.1
    wt.step_rk4_curved(P, Q, coef, ws, dt, nsteps, eps_KO=eps, bc3d=bc, metric=True)
    slabs = [S.Slab(ctx, r, N, M, **kw, bg_kind=wt.BG_ADM_PERTURBED, bg_params=prm, mu=ws.mu)
             for r in S.partition(M[2], nslabs, periodic, depth=6)]
    for s in slabs:
        wt.initial_data(s.mesh, wt.IC_GAUSSIANS, ic, s.Phi)
    with pytest.raises(ValueError):               # the flux halo is one layer deep
        S.step(slabs, S.LocalHalo(slabs), dt, 1, bc)
    S.step_ko(slabs, S.LocalStateHalo(slabs), dt, nsteps, eps, bc)
    Ps = torch.cat([s.owned(s.Phi) for s in slabs])
    Qs = torch.cat([s.owned(s.Pi) for s in slabs])
    assert float(P.abs().max()) < 3.0 and float(Q.abs().max()) < 50.0   # a bounded solution, not a blow-up
    dP = float((Ps - P).abs().max()) / float(P.abs().max())
    dQ = float((Qs - Q).abs().max()) / float(Q.abs().max())
    tol = 1e-13 if prec == wt.WT_F64 else 1e-6
    assert dP <= tol and dQ <= tol, (dP, dQ)
    for s in slabs:
        s.close()
    assert not ctx.nonfinite()


def test_face_halo_errors_and_size(wt, ctx):
    import torch
    g = wt.Mesh.slab(ctx, 6, (2, 3, 5), 1, 3)
    ws = wt.make_wave3d_workspace(g)
    c = wt.sample_background3d(g, wt.BG_MINKOWSKI)
    P, Q = g.zeros(), g.zeros()
    with pytest.raises(wt.WaveToyError):          # nothing to size before a stage has run
        wt.halo_face_size(ws)
    with pytest.raises(wt.WaveToyError):          # the slab has layers 0..2
        wt.rk4_stage_curved_layers(P, Q, c, ws, 1e-3, 0, 1, 2, 2, metric=True)
    wt.rk4_stage_curved_layers(P, Q, c, ws, 1e-3, 0, 1, 1, 1, metric=True)
    n = wt.halo_face_size(ws)
    assert n == 6 * 6 ** 2 * 4                    # Phi + three flux components on the faces of 6 elements
    buf = torch.empty(n, dtype=torch.float64, device="cuda")
    with pytest.raises(wt.WaveToyError):
        wt.halo_face_copy(ws, P, 0, 1, 3, buf, True)   # faces 4 (-z) and 5 (+z) only
    with pytest.raises(wt.WaveToyError):
        wt.halo_face_copy(ws, P, 0, 3, 5, buf, True)
    wt.halo_face_copy(ws, P, 0, 1, 5, buf, True)
