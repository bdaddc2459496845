"""Device-side diagnostics and snapshots: the slice, L2 and energy samples of
evolve_curved_device equal what the host-copy loop (evolve_curved_host, the
shape of evolve3d) gives for the same evolution, and a snapshot written and read
back restores the state bit for bit."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def setup(wt, ctx, prec=0):
    g = wt.Mesh.uniform_hex(ctx, 6, 2, outer_tag=7, warp_A=0.0, precision=prec)
    p = wt.workloads.adm_params(4)
    c = wt.sample_background3d(g, wt.BG_ADM_PERTURBED, p)
    ws = wt.make_wave3d_workspace(g)
    Phi, Pi = g.zeros(), g.zeros()
    cc, a, w = wt.workloads.pulses(4, 2)
    wt.initial_data(g, wt.IC_GAUSSIANS, wt.gaussian_params(cc, a, w), Phi)
    dt = 0.2 * g.min_spacing() / wt.workloads.max_speed(p)
    return g, c, ws, Phi, Pi, dt


def test_device_samples_equal_host_loop(wt, ctx):
    g, c, ws, Phi, Pi, dt = setup(wt, ctx)
    bc = wt.make_bc3d([wt.BC_SOMMERFELD] * 6)
    P0, Q0 = Phi.cpu().numpy().copy(), Pi.cpu().numpy().copy()
    res = wt.evolve_curved_device(Phi, Pi, c, ws, dt, 4, 3, bc3d=bc, metric=True, slice_yz=(0.5, 0.5))
    nodes, xs = wt.slice_nodes(g, 0.5, 0.5)
    assert len(nodes) == len(res["xs_line"]) > 0 and np.all(np.diff(xs) > 0)  # a shared node appears once
    # the same evolution through the host-copy loop, one sample at a time
    Hd = g.get("Hd")
    ws2 = wt.make_wave3d_workspace(g)
    Ph, Qh = P0.copy(), Q0.copy()
    for n in range(3):
        E = np.zeros(1)
        wt.evolve_curved_host(Ph, Qh, c, ws2, dt, 4, 1, bc3d=bc, metric=True, energy=E)
        assert np.max(np.abs(res["Phis"][:, n] - Ph[nodes])) == 0.0
        assert np.max(np.abs(res["Pis"][:, n] - Qh[nodes])) == 0.0
        assert abs(res["l2_err"][n] - np.sqrt(np.sum(Ph ** 2 * Hd))) <= 1e-12 * res["l2_err"][n]
        assert abs(res["energy"][n] - E[0]) <= 1e-12 * abs(E[0])
    assert np.array_equal(Phi.cpu().numpy(), Ph) and np.array_equal(Pi.cpu().numpy(), Qh)


@pytest.mark.parametrize("prec", [0, 1])
def test_snapshot_round_trip(wt, ctx, tmp_path, prec):
    import torch
    g, c, ws, Phi, Pi, dt = setup(wt, ctx, prec)
    Pi.copy_(torch.randn_like(Pi))
    path = tmp_path / "state.wtsnap"
    wt.snapshot_save(str(path), Phi, Pi, g, t=1.25)
    A, B = g.zeros(), g.zeros()
    assert wt.snapshot_load(str(path), A, B, g) == 1.25
    assert torch.equal(A, Phi) and torch.equal(B, Pi)
    other = wt.Mesh.uniform_hex(ctx, 4, 3, precision=prec)
    with pytest.raises(wt.WaveToyError):
        wt.snapshot_load(str(path), other.zeros(), other.zeros(), other)
    with pytest.raises(wt.WaveToyError):
        wt.gather_nodes(Phi, [g.nn], g)
