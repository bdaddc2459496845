"""GPU: the fused RK4 stage kernel (FP64, n = 8) against the two-kernel stages and
the oracle.

The fused step runs K1_0, then three launches that each do the divergence half
of stage s and the gradient half of stage s + 1 on every element, then K2_3
(the integrator fused into the right-hand side, the reference's IDEAS.md:48-50;
arithmetic of wave3d_curved_rhs!, src/wave3d_curved.jl:205-258).  Each half
repeats the arithmetic of its two-kernel counterpart in the same order, so the
fused and the two-kernel steps must agree bit for bit; the fused step (the
default, so also what the other FP64 n = 8 stepping tests run) is held to the
oracle at <= 1e-12.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL64 = 1e-12


def rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def host(x):
    return x.detach().double().cpu().numpy()


def _setup(wt, ctx, O, M, periodic=False, outer_tag=7, kind=2, params=None, seed=5):
    g = wt.Mesh.uniform_hex(ctx, 8, M, periodic=periodic, outer_tag=outer_tag, warp_A=0.05)
    o = O.OracleMesh(8, M, A=0.05, periodic=periodic, outer_tag=outer_tag)
    p = wt.workloads.adm_params(seed) if params is None else params
    x, y, z = o.coords()
    Phi = wt.workloads.gaussian_field(x, y, z, *wt.workloads.pulses(seed, 3))
    Pi = 0.2 * np.sin(2 * np.pi * x) * Phi
    return g, o, p, Phi, Pi


def _run(wt, ctx, g, kind, p, Phi, Pi, dt, nsteps, bc, fused, split=(2,)):
    import torch
    c = wt.sample_background3d(g, kind, p)
    ws = wt.make_wave3d_workspace(g)
    ws.set_fused(fused)
    P = torch.tensor(Phi, dtype=torch.float64, device="cuda")
    Q = torch.tensor(Pi, dtype=torch.float64, device="cuda")
    done = 0
    for k in list(split) + [nsteps]:  # some steps launched one by one, the rest through the graph replay
        k = min(k, nsteps) - done
        if k > 0:
            wt.step_rk4_curved(P, Q, c, ws, dt, k, bc3d=bc, metric=True)
            done += k
    ctx.synchronize()
    assert not ctx.nonfinite()
    return P, Q, c


@pytest.mark.parametrize("M,kinds,exc", [
    ((6, 6, 6), [2] * 6, 0),     # 216 elements: more than one per SM, both ring stages cycle
    (3, [2] * 6, 0),             # 27 elements: fewer CTAs than SMs
    ((8, 8, 6), [4] * 6, 0),     # full-Dirichlet data on every outer face
    ((8, 8, 6), [1] * 6, 8),     # Dirichlet characteristic data, -z faces excised
])
def test_fused_equals_two_kernel_stages_bitwise(wt, ctx, O, M, kinds, exc):
    import torch
    g, o, p, Phi, Pi = _setup(wt, ctx, O, M)
    if exc:
        bd = o.get("bdry").copy()
        bd[4::6][bd[4::6] != 0] = exc
        o.set_bdry(bd)
        g.set_bdry(bd)
    rng = np.random.default_rng(7)
    data = [torch.tensor(rng.standard_normal(o.nn), device="cuda") for _ in range(5)]
    bc = wt.make_bc3d(kinds, gPhi=data[0], gPi=data[1], gDx=data[2], gDy=data[3], gDz=data[4], excision_tag=exc)
    dt = 0.2 * o.min_spacing() / wt.workloads.max_speed(p)
    Pf, Qf, _ = _run(wt, ctx, g, 2, p, Phi, Pi, dt, 7, bc, True)
    Pu, Qu, _ = _run(wt, ctx, g, 2, p, Phi, Pi, dt, 7, bc, False)
    assert torch.equal(Pf, Pu) and torch.equal(Qf, Qu)


def test_fused_matches_oracle_many_steps(wt, ctx, O):
    """30 fused steps (2 launched one by one, 28 replayed) of three pulses on the warped ADM
    background with Sommerfeld faces on 4 x 5 x 6 elements, against the oracle's classic RK4."""
    g, o, p, Phi, Pi = _setup(wt, ctx, O, (4, 5, 6), seed=11)
    dt = 0.2 * o.min_spacing() / wt.workloads.max_speed(p)
    bc = wt.make_bc3d([2] * 6)
    P, Q, _ = _run(wt, ctx, g, 2, p, Phi, Pi, dt, 30, bc, True)
    Po, Qo = o.evolve_curved(o.background(2, p), Phi, Pi, dt, 30, bc=O.make_bc([2] * 6), use_metric=True)
    assert rel(host(P), Po) < TOL64 and rel(host(Q), Qo) < TOL64


def test_fused_periodic_equals_two_kernel_stages(wt, ctx, O):
    """A periodic warped cube (no outer face, every face a SAT face)."""
    import torch
    g, o, p, Phi, Pi = _setup(wt, ctx, O, 4, periodic=True, outer_tag=0)
    dt = 0.2 * o.min_spacing() / wt.workloads.max_speed(p)
    Pf, Qf, _ = _run(wt, ctx, g, 2, p, Phi, Pi, dt, 5, None, True)
    Pu, Qu, _ = _run(wt, ctx, g, 2, p, Phi, Pi, dt, 5, None, False)
    assert torch.equal(Pf, Pu) and torch.equal(Qf, Qu)


@pytest.mark.parametrize("kind", [4, 5])
def test_fused_time_dependent_background(wt, ctx, O, kind):
    """Gauge wave / sine shift re-sampled before each launch whose gradient half reads the
    coefficients: equal to the two-kernel stages, the coefficients' time advanced by the steps."""
    import torch
    g, o, _, Phi, Pi = _setup(wt, ctx, O, 3)
    A, d, t0 = 0.15, 1.0, 0.05
    dt = 0.2 * o.min_spacing() / ((1 + A) / (1 - A))
    bc = wt.make_bc3d([2] * 6)
    Pf, Qf, cf = _run(wt, ctx, g, kind, (A, d, t0), Phi, Pi, dt, 6, bc, True)
    Pu, Qu, cu = _run(wt, ctx, g, kind, (A, d, t0), Phi, Pi, dt, 6, bc, False)
    assert torch.equal(Pf, Pu) and torch.equal(Qf, Qu)
    assert abs(cf.time - (t0 + 6 * dt)) < 1e-14 and cf.time == cu.time


def test_fused_path_taken(wt, ctx, O):
    """One step is five launches through the fused path (K1_0, three fused stages, K2_3) and eight
    through the two-kernel stages; the profile sees the fused launches."""
    import torch
    g, o, p, Phi, Pi = _setup(wt, ctx, O, 2)
    c = wt.sample_background3d(g, 2, p)
    ws = wt.make_wave3d_workspace(g)
    P = torch.tensor(Phi, device="cuda")
    Q = torch.tensor(Pi, device="cuda")
    bc = wt.make_bc3d([2] * 6)
    counts = []
    for fused in (True, False):
        ws.set_fused(fused)
        wt.step_rk4_curved(P, Q, c, ws, 1e-4, 1, bc3d=bc, metric=True)  # allocates the second flux buffer
        ctx.synchronize()
        n0 = ctx.launch_count()
        ctx.profile(True)
        wt.step_rk4_curved(P, Q, c, ws, 1e-4, 1, bc3d=bc, metric=True)
        ctx.profile(False)
        prof = ctx.profile_read()
        counts.append((ctx.launch_count() - n0, [n for _, n in prof]))
    assert counts[0] == (5, [1, 1, 3])
    assert counts[1] == (8, [4, 4, 0])


@pytest.mark.parametrize("M,periodic", [((1, 1, 1), False), ((1, 1, 1), True), ((1, 3, 2), False), ((2, 1, 3), True)])
def test_fused_degenerate_meshes(wt, ctx, O, M, periodic):
    """One element (every face outer, or its own neighbour on every face of a periodic cube) and
    one-element-thick meshes: fused = two-kernel bit for bit, and the fused step against the oracle."""
    import torch
    g, o, p, Phi, Pi = _setup(wt, ctx, O, M, periodic=periodic, outer_tag=0 if periodic else 7, seed=13)
    bc = None if periodic else wt.make_bc3d([2] * 6)
    dt = 0.2 * o.min_spacing() / wt.workloads.max_speed(p)
    Pf, Qf, _ = _run(wt, ctx, g, 2, p, Phi, Pi, dt, 5, bc, True)
    Pu, Qu, _ = _run(wt, ctx, g, 2, p, Phi, Pi, dt, 5, bc, False)
    assert torch.equal(Pf, Pu) and torch.equal(Qf, Qu)
    Po, Qo = o.evolve_curved(o.background(2, p), Phi, Pi, dt, 5, bc=None if periodic else O.make_bc([2] * 6),
                             use_metric=True)
    assert rel(host(Pf), Po) < TOL64 and rel(host(Qf), Qo) < TOL64
