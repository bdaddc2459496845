"""Failure detection without a GPU fault: the pipelined kernels' bounded waits
report WT_ETIMEOUT through the context status word when they give up (here a
one-thread self-test of the same wait on an mbarrier nothing arrives at), a
non-finite state is flagged by the RK4 epilogue, and the context keeps working
afterwards."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_bounded_wait_gives_up_and_context_survives(wt, ctx):
    import torch
    ctx.selftest_wait(True)                      # the phase completes: no error
    with pytest.raises(wt.WaveToyError) as ei:
        ctx.selftest_wait(False, polls=1 << 12)  # nothing arrives: the wait gives up
    assert ei.value.code == -6
    assert not ctx.nonfinite()                   # reported once, then cleared
    g = wt.Mesh.uniform_hex(ctx, 8, 2, outer_tag=7, warp_A=0.05)
    c = wt.sample_background3d(g, wt.BG_ADM_PERTURBED, wt.workloads.adm_params(1))
    ws = wt.make_wave3d_workspace(g)
    P = torch.randn(g.nn, dtype=torch.float64, device="cuda")
    Q = torch.zeros_like(P)
    wt.step_rk4_curved(P, Q, c, ws, 1e-3, 3, bc3d=wt.make_bc3d([2] * 6), metric=True)
    assert torch.isfinite(P).all() and not ctx.nonfinite()
    with pytest.raises(wt.WaveToyError):
        ctx.selftest_wait(True, polls=0)


def test_nonfinite_state_is_flagged(wt, ctx):
    import torch
    g = wt.Mesh.uniform_hex(ctx, 8, 2, outer_tag=7, warp_A=0.05)
    c = wt.sample_background3d(g, wt.BG_ADM_PERTURBED, wt.workloads.adm_params(1))
    ws = wt.make_wave3d_workspace(g)
    P = torch.zeros(g.nn, dtype=torch.float64, device="cuda")
    P[17] = float("nan")
    Q = torch.zeros_like(P)
    wt.step_rk4_curved(P, Q, c, ws, 1e-3, 1, bc3d=wt.make_bc3d([2] * 6), metric=True)
    assert ctx.nonfinite()
    assert not ctx.nonfinite()                   # cleared by the read
    Ph = np.zeros(g.nn)
    Ph[5] = np.inf
    with pytest.raises(wt.WaveToyError) as ei:
        wt.evolve_curved_host(Ph, np.zeros(g.nn), c, ws, 1e-3, 1, 1, bc3d=wt.make_bc3d([2] * 6), metric=True)
    assert ei.value.code == -5
