"""wt_rhs_curved_noalloc: the conservative RHS with its scratch in the library's
fixed device array instead of a workspace.

Each case calls the allocation-free entry point twice in a row, on different
inputs, through the C ABI and compares both results with wt_rhs_curved on the
same inputs (tolerance 1e-12 relative L2, as for the other RHS parity tests).
The second call runs on whatever the first left in the shared array.
This file is collected last, so it also runs after the rest of the GPU suite
has used the same context.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL64 = 1e-12


def rel(a, b):
    a = a.detach().double().cpu().numpy()
    b = b.detach().double().cpu().numpy()
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def fields(mesh, seed):
    import torch
    g = torch.Generator(device="cpu").manual_seed(seed)
    Phi = torch.randn(mesh.nn, generator=g, dtype=torch.float64).cuda()
    Pi = torch.randn(mesh.nn, generator=g, dtype=torch.float64).cuda()
    return Phi, Pi


@pytest.mark.parametrize("case", ["n8_max_size_sommerfeld", "n5_affine_dirichlet_ko"])
def test_noalloc_matches_workspace_rhs_twice(wt, ctx, case):
    import torch
    if case == "n8_max_size_sommerfeld":
        # 8^3 elements of n = 8: exactly the node limit; FP64 curvilinear, so the
        # pipelined tensor-core kernels run
        mesh = wt.Mesh.uniform_hex(ctx, 8, (8, 8, 8), 0.0, 1.0, outer_tag=7, warp_A=0.05)
        assert mesh.nn == wt.NOALLOC_MAX_NODES
        bc = wt.make_bc3d([wt.BC_SOMMERFELD] * 6)
        metric, eps = True, 0.0
    else:
        mesh = wt.Mesh.uniform_hex(ctx, 5, (3, 4, 2), 0.0, 1.0, outer_tag=0)
        gen = torch.Generator(device="cpu").manual_seed(5)
        gd = [torch.randn(mesh.nn, generator=gen, dtype=torch.float64).cuda() for _ in range(5)]
        bc = wt.make_bc3d([wt.BC_DIRICHLET] * 6, gPhi=gd[0], gPi=gd[1], gDx=gd[2], gDy=gd[3], gDz=gd[4])
        metric, eps = False, 0.1
    coef = wt.sample_background3d(mesh, wt.BG_ADM_PERTURBED, wt.workloads.adm_params(7))
    ws = wt.make_wave3d_workspace(mesh)
    ref_P, ref_Q = mesh.zeros(), mesh.zeros()
    out_P, out_Q = mesh.zeros(), mesh.zeros()
    free = []
    for call, seed in enumerate((101, 202)):
        Phi, Pi = fields(mesh, seed)
        wt.wave3d_curved_rhs(ref_P, ref_Q, Phi, Pi, coef, ws, eps_KO=eps, bc3d=bc, metric=metric)
        out_P.fill_(float("nan"))
        out_Q.fill_(float("nan"))
        torch.cuda.synchronize()
        before = torch.cuda.mem_get_info()[0]
        wt.wave3d_curved_rhs_noalloc(out_P, out_Q, Phi, Pi, coef, eps_KO=eps, mu=ws.mu, bc3d=bc, metric=metric)
        torch.cuda.synchronize()
        free.append((before, torch.cuda.mem_get_info()[0]))
        assert torch.isfinite(out_P).all() and torch.isfinite(out_Q).all(), f"call {call}"
        assert rel(out_P, ref_P) < TOL64, f"call {call}"
        assert rel(out_Q, ref_Q) < TOL64, f"call {call}"
    # after the first call on the device (set-up) a call takes no device memory;
    # any device allocation would take at least 2 MiB
    before, after = free[1]
    assert before - after < 2 << 20
    assert not ctx.nonfinite()


def test_noalloc_rejects_meshes_above_the_limit(wt, ctx):
    mesh = wt.Mesh.uniform_hex(ctx, 8, (8, 8, 9), 0.0, 1.0, outer_tag=7, warp_A=0.05)
    assert mesh.nn > wt.NOALLOC_MAX_NODES
    coef = wt.sample_background3d(mesh, wt.BG_ADM_PERTURBED, wt.workloads.adm_params(7))
    P, Q = mesh.zeros(), mesh.zeros()
    with pytest.raises(wt.WaveToyError) as ei:
        wt.wave3d_curved_rhs_noalloc(P, Q, P, Q, coef, metric=True)
    assert ei.value.code == -1
    assert "at most 262144" in str(ei.value)


def test_noalloc_rejects_non_finite_mu(wt, ctx):
    mesh = wt.Mesh.uniform_hex(ctx, 5, (2, 2, 2), 0.0, 1.0, outer_tag=0)
    coef = wt.sample_background3d(mesh, wt.BG_ADM_PERTURBED, wt.workloads.adm_params(7))
    P, Q = mesh.zeros(), mesh.zeros()
    for mu in (float("inf"), float("nan"), 0.0, -1.0):
        with pytest.raises(wt.WaveToyError) as ei:
            wt.wave3d_curved_rhs_noalloc(P, Q, P, Q, coef, eps_KO=0.1, mu=mu)
        assert ei.value.code == -1
        assert "positive and finite" in str(ei.value)
