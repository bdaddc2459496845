"""Batched solves (wt_batch_*): many solves of uneven element counts, orders and
precisions advanced together must give what each gives when stepped alone
with wt_step_rk4_curved (<= 1e-12 relative L2 for FP64 members, <= 1e-6 for
FP32 members, which run the same kernels), also after members leave and join.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel(a, b):
    a = a.double().cpu().numpy()
    b = b.double().cpu().numpy()
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


class Solve:
    """One member: mesh, ADM background, pulse data, a workspace for the batch
    and a second workspace + state copy stepped alone."""

    def __init__(self, wt, ctx, N, M, seed, precision=0, form=None, amp=0.1):
        W = wt.workloads
        self.mesh = wt.Mesh.uniform_hex(ctx, N, M, outer_tag=7, warp_A=0.05, precision=precision)
        if form is not None:
            self.mesh.set_fp32_form(form)
        p = W.adm_params(seed, amp)
        self.coef = wt.sample_background3d(self.mesh, wt.BG_ADM_PERTURBED, p)
        self.ws, self.ws_alone = wt.make_wave3d_workspace(self.mesh), wt.make_wave3d_workspace(self.mesh)
        self.Phi, self.Pi = self.mesh.zeros(), self.mesh.zeros()
        c, a, w = W.pulses(seed, 2, amp=(0.5, 1.0), width=(0.05, 0.15))
        wt.initial_data(self.mesh, wt.IC_GAUSSIANS, wt.gaussian_params(c, a, w), self.Phi)
        self.Pa, self.Qa = self.Phi.clone(), self.Pi.clone()
        self.dt = 0.2 * self.mesh.min_spacing() / W.max_speed(p)
        self.bc = wt.make_bc3d([wt.BC_SOMMERFELD] * 6)
        self.tol = 1e-12 if precision == 0 else 1e-6

    def step_alone(self, wt, n):
        wt.step_rk4_curved(self.Pa, self.Qa, self.coef, self.ws_alone, self.dt, n, bc3d=self.bc, metric=True)

    def check(self):
        assert rel(self.Phi, self.Pa) <= self.tol and rel(self.Pi, self.Qa) <= self.tol


def test_batch_matches_solves_stepped_alone(wt, ctx):
    specs = [(4, 3, 11, 0, None), (6, 2, 12, 0, None), (8, 2, 13, 0, None), (8, (3, 2, 2), 14, 0, None),
             (8, 2, 15, 1, wt.FP32_BF16X3), (6, 3, 16, 1, None), (8, 2, 17, 1, wt.FP32_CUDA_CORES),
             (5, 2, 18, 0, None)]
    solves = [Solve(wt, ctx, N, M, seed, prec, form, amp=0.15 * (k % 3) / 2) for k, (N, M, seed, prec, form)
              in enumerate(specs)]
    batch = wt.Batch(ctx)
    slots = [batch.add(s.Phi, s.Pi, s.coef, s.ws, s.dt, s.bc) for s in solves]
    # the RK4 path does not read the FP64 set-up geometry; releasing it must not matter
    solves[4].mesh.release_setup_geometry()
    with pytest.raises(wt.WaveToyError):
        solves[4].mesh.min_spacing()
    nsolves, nodes, ngroups = batch.info()
    assert nsolves == len(solves) and nodes == sum(s.mesh.nn for s in solves)
    groups = batch.groups()
    assert ngroups == len(groups) >= 5
    assert any(g[2] == 1 and g[1] == 0 for g in groups) and any(g[2] == 1 and g[1] == 1 for g in groups)
    batch.step(7)
    for s in solves:
        s.step_alone(wt, 7)
    for s in solves:
        s.check()
    # members leave and join; the others carry on unchanged
    batch.remove(slots[1])
    batch.remove(slots[4])
    extra = Solve(wt, ctx, 4, 2, 19)
    batch.add(extra.Phi, extra.Pi, extra.coef, extra.ws, extra.dt, extra.bc)
    batch.step(5)
    for k, s in enumerate(solves):
        if k not in (1, 4):
            s.step_alone(wt, 5)
            s.check()
    extra.step_alone(wt, 5)
    extra.check()
    E = wt.wave3d_energy(solves[4].Phi, solves[4].Pi, solves[4].coef, solves[4].ws, metric=True)
    assert np.isfinite(E) and E > 0
    assert not ctx.nonfinite()
    batch.close()


def test_batch_autotune_off_gives_same_results(wt, ctx):
    a = Solve(wt, ctx, 4, 4, 21)
    b = Solve(wt, ctx, 4, 4, 21)
    b1, b2 = wt.Batch(ctx, autotune=True), wt.Batch(ctx, autotune=False)
    b1.add(a.Phi, a.Pi, a.coef, a.ws, a.dt, a.bc)
    b2.add(b.Phi, b.Pi, b.coef, b.ws, b.dt, b.bc)
    b1.step(4)
    b2.step(4)
    assert b2.groups()[0][3] == 0
    assert rel(a.Phi, b.Phi) <= 1e-12 and rel(a.Pi, b.Pi) <= 1e-12


def test_batch_rejects_bad_members(wt, ctx):
    s = Solve(wt, ctx, 4, 2, 31)
    batch = wt.Batch(ctx)
    with pytest.raises(wt.WaveToyError):
        batch.add(s.Phi, s.Pi, s.coef, s.ws, -1.0, s.bc)
    batch.add(s.Phi, s.Pi, s.coef, s.ws, s.dt, s.bc)
    with pytest.raises(wt.WaveToyError):  # one workspace serves one member
        batch.add(s.Pa, s.Qa, s.coef, s.ws, s.dt, s.bc)
    with pytest.raises(wt.WaveToyError):
        batch.remove(7)


@pytest.mark.parametrize("variant", [-1, 2])
def test_batch_members_against_oracle(wt, ctx, O, variant):
    """Members of one mixed batch (n = 4, 6, 8; FP64 and the default compensated FP32
    form; groups running as parallel graph branches) against the Float64 oracle after
    60 steps: FP64 <= 1e-12, compensated FP32 <= 1e-5 relative L2.  variant: the
    autotuner's choice (-1) or the pipelined n = 4, 6 kernels (2)."""
    import torch
    W = wt.workloads
    specs = [(4, 3, 41, 0), (6, 2, 42, 1), (8, 2, 43, 1), (8, 2, 44, 0), (6, 2, 45, 0), (4, 3, 46, 1)]
    members = []
    batch = wt.Batch(ctx)
    batch.set_variant(variant, variant)
    bc = wt.make_bc3d([wt.BC_SOMMERFELD] * 6)
    for N, M, seed, prec in specs:
        g = wt.Mesh.uniform_hex(ctx, N, M, outer_tag=7, warp_A=0.05, precision=prec)
        p = W.adm_params(seed, 1.0)
        coef = wt.sample_background3d(g, wt.BG_ADM_PERTURBED, p)
        ws = wt.make_wave3d_workspace(g)
        c, a, w = W.pulses(seed, 2, amp=(0.5, 1.0), width=(0.08, 0.15))
        Phi, Pi = g.zeros(), g.zeros()
        wt.initial_state(ws, wt.IC_GAUSSIANS, wt.gaussian_params(c, a, w), Phi, Pi)
        dt = 0.2 * g.min_spacing() / W.max_speed(p)
        batch.add(Phi, Pi, coef, ws, dt, bc)
        members.append((N, M, seed, prec, p, (c, a, w), dt, g, coef, ws, Phi, Pi))
    assert batch.info()[2] == 6  # one group per (n, precision)
    batch.step(60)
    for N, M, seed, prec, p, pul, dt, g, coef, ws, Phi, Pi in members:
        o = O.OracleMesh(N, M, A=0.05, outer_tag=7)
        x, y, z = o.coords()
        P0 = W.gaussian_field(x, y, z, *pul)
        Po, Qo = o.evolve_curved(o.background(2, p), P0, np.zeros_like(P0), dt, 60, bc=O.make_bc([2] * 6),
                                 use_metric=True)
        err = np.linalg.norm(np.concatenate([Phi.double().cpu().numpy(), Pi.double().cpu().numpy()]) -
                             np.concatenate([Po, Qo])) / np.linalg.norm(np.concatenate([Po, Qo]))
        assert err <= (1e-12 if prec == 0 else 1e-5), (N, M, prec, err)
    assert not ctx.nonfinite()
    batch.close()


@pytest.mark.parametrize("branches", [True, False])
def test_batch_time_dependent_backgrounds(wt, ctx, branches):
    """Gauge-wave and sine-shift members (re-sampled at every stage inside the batch
    graph) beside a static member: each matches its solve stepped alone with
    wt_step_rk4_curved, and each background's time advances with the steps.  Both with
    the groups as parallel graph branches and with one group (FP64 members only)."""
    specs = [(6, 2, wt.BG_GAUGE_WAVE, 0), (8, 2, wt.BG_SINE_SHIFT, 1), (4, 3, None, 0)]
    if not branches:
        specs = [(6, 2, wt.BG_GAUGE_WAVE, 0), (6, 3, wt.BG_SINE_SHIFT, 0)]
    batch = wt.Batch(ctx)
    bc = wt.make_bc3d([wt.BC_SOMMERFELD] * 6)
    members = []
    for k, (N, M, kind, prec) in enumerate(specs):
        g = wt.Mesh.uniform_hex(ctx, N, M, outer_tag=7, warp_A=0.05, precision=prec)
        if kind is None:
            prm = wt.workloads.adm_params(50 + k)
            mk = lambda: wt.sample_background3d(g, wt.BG_ADM_PERTURBED, prm)
            speed = wt.workloads.max_speed(prm)
        else:
            A, t0 = 0.1 + 0.02 * k, 0.03 * k
            mk = lambda: wt.sample_background3d(g, kind, (A, 1.0, t0))
            speed = (1 + A) / (1 - A)
        cb, ca = mk(), mk()
        ws, ws_alone = wt.make_wave3d_workspace(g), wt.make_wave3d_workspace(g)
        c, a, w = wt.workloads.pulses(60 + k, 2, amp=(0.5, 1.0), width=(0.08, 0.15))
        P, Q = g.zeros(), g.zeros()
        wt.initial_state(ws, wt.IC_GAUSSIANS, wt.gaussian_params(c, a, w), P, Q)
        Pa, Qa = P.clone(), Q.clone()
        dt = 0.2 * g.min_spacing() / speed
        batch.add(P, Q, cb, ws, dt, bc)
        members.append((kind, prec, cb, ca, ws_alone, P, Q, Pa, Qa, dt))
    assert (batch.info()[2] > 1) == branches
    for n in (3, 5):
        batch.step(n)
        for kind, prec, cb, ca, wsa, P, Q, Pa, Qa, dt in members:
            wt.step_rk4_curved(Pa, Qa, ca, wsa, dt, n, bc3d=bc, metric=True)
    for kind, prec, cb, ca, wsa, P, Q, Pa, Qa, dt in members:
        tol = 1e-12 if prec == 0 else 1e-6
        assert rel(P, Pa) <= tol and rel(Q, Qa) <= tol, (kind, rel(P, Pa), rel(Q, Qa))
        if kind is not None:
            assert abs(cb.time - ca.time) < 1e-14 and cb.time > 0.2 * dt
            np.testing.assert_allclose(cb.get(), ca.get(), rtol=0, atol=1e-13)
    assert not ctx.nonfinite()
    batch.close()


@pytest.mark.parametrize("prec,form", [(0, None), (1, None), (1, "cuda")])
def test_batch_pipelined_kernels_bitwise(wt, ctx, prec, form):
    """The persistent cp.async-pipelined n = 4, 6 kernels (launch variant 2) against the generic
    kernels (variant 0): bit-identical states after 7 steps, for FP64, the compensated FP32 form and
    plain FP32; the 512- and 2197-element members make each persistent CTA loop over several
    groups of tiles, the small ones leave most of the grid idle."""
    import torch
    specs = [(6, 8, 51, 0.1), (4, 13, 52, 0.05), (6, 3, 53, 0.15), (4, 2, 54, 0.0)]
    fform = {None: None, "cuda": wt.FP32_CUDA_CORES}[form]
    runs = []
    for var in (0, 2):
        solves = [Solve(wt, ctx, N, M, seed, prec, fform if prec else None, amp) for N, M, seed, amp in specs]
        b = wt.Batch(ctx)
        b.set_variant(var, var)
        for s in solves:
            b.add(s.Phi, s.Pi, s.coef, s.ws, s.dt, s.bc)
        b.step(2)
        b.step(5)
        assert all(g[3] == var | (var << 2) for g in b.groups() if not g[2])
        runs.append(solves)
        b.close()
    for a, c in zip(*runs):
        assert torch.equal(a.Phi, c.Phi) and torch.equal(a.Pi, c.Pi)
    assert not ctx.nonfinite()
