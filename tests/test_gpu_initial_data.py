"""GPU parity of the device-side set-up that every solve starts from: the initial
data families of wt_initial_data and the CFL spacing of wt_mesh_min_spacing,
against the oracle's restatements evaluated at the oracle's own node coordinates.

Initial data (FP64 meshes, <= 1e-12 relative L2; FP32 meshes, the FP64 field
rounded once, <= 1e-7):
  * eigenmode_cartesian!  (src/wave.jl:163-185), at t = 0 and t = 0.37;
  * the :gaussian IC      (src/evolve.jl:1260-1263), summed seeded pulses;
  * outgoing_pulse!       (src/wave.jl:292-323), including the node at r = 0
    (the sinhc Taylor branch, src/wave.jl:242-250);
  * the constant-shift plane wave Phi_e, Pi_e (src/evolve.jl:1119-1120);
  * eigenmode_radial!     (src/wave.jl:207-226), including r = 0.
Spacing: _min_node_spacing_3d (src/evolve.jl:60-69) over all three reference
directions, on warped, periodic and multi-patch meshes (<= 1e-14 relative), and
the CFL step dt = cfl * dx_min / max_speed (src/evolve.jl:1209-1213) built on it.
"""
import math

import numpy as np
import pytest

from test_patch_meshes import KINDS, oracle_from

pytestmark = pytest.mark.gpu


def rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def host(x):
    return x.detach().double().cpu().numpy()


def cases(wt):
    c, a, w = wt.workloads.pulses(21, 4, amp=(0.5, 1.0), width=(0.05, 0.15), centre=(0.25, 0.75))
    pulses = [(c[k][0], c[k][1], c[k][2], a[k], w[k]) for k in range(len(a))]
    k = 2 * math.pi
    s = 0.1 + 0.05 - 0.2   # constant shift bx + by + bz
    om = -k * s + k * math.sqrt(3.0)
    return [
        ("eigenmode_cartesian", wt.IC_EIGENMODE_CARTESIAN,
         [1.3, math.pi, 2 * math.pi, math.pi, math.sqrt(6) * math.pi, 0.0, 1.0], (0.0, 0.37),
         lambda O, x, y, z, t: O.ic_eigenmode_cartesian(x, y, z, t, 1.3, math.pi, 2 * math.pi, math.pi,
                                                        math.sqrt(6) * math.pi, 0.0, 1.0)),
        ("gaussians", wt.IC_GAUSSIANS, wt.gaussian_params(c, a, w), (0.0,),
         lambda O, x, y, z, t: O.ic_gaussians(x, y, z, pulses)),
        # centred on a node of the cube (r = 0 is a node)
        ("outgoing_pulse", wt.IC_OUTGOING_PULSE, [0.8, 0.3, 0.07, 0.5, 0.5, 0.5], (0.0, 0.11),
         lambda O, x, y, z, t: O.ic_outgoing_pulse(x, y, z, t, 0.8, 0.3, 0.07, 0.5, 0.5, 0.5)),
        ("plane_wave", wt.IC_PLANE_WAVE, [k, om, s], (0.0, 0.23),
         lambda O, x, y, z, t: O.ic_plane_wave(x, y, z, t, k, om, s)),
        ("eigenmode_radial", wt.IC_EIGENMODE_RADIAL, [1.1, 0.9, 2.0, 0.5, 0.5, 0.5], (0.0, 0.41),
         lambda O, x, y, z, t: O.ic_eigenmode_radial(x, y, z, t, 1.1, 0.9, 2.0, 0.5, 0.5, 0.5)),
    ]


@pytest.mark.parametrize("which", range(5))
@pytest.mark.parametrize("prec", [0, 1])
def test_initial_data_matches_oracle(wt, ctx, O, which, prec):
    # 4 elements per axis: element corners at 0.25, 0.5, 0.75, so (0.5, 0.5, 0.5) is a node
    g = wt.Mesh.uniform_hex(ctx, 6, (4, 4, 4), 0.0, 1.0, warp_A=0.05, outer_tag=7, precision=prec)
    o = O.OracleMesh(6, (4, 4, 4), A=0.05, outer_tag=7)
    name, kind, params, times, ref = cases(wt)[which]
    x, y, z = o.coords()
    if kind in (wt.IC_OUTGOING_PULSE, wt.IC_EIGENMODE_RADIAL):
        assert np.min((x - 0.5) ** 2 + (y - 0.5) ** 2 + (z - 0.5) ** 2) == 0.0
    tol = 1e-12 if prec == 0 else 1e-7
    for t in times:
        u, ut = g.zeros(), g.zeros()
        wt.initial_data(g, kind, params, u, ut, t=t)
        uo, uto = ref(O, x, y, z, t)
        assert np.all(np.isfinite(host(u))) and np.all(np.isfinite(host(ut))), name
        assert rel(host(u), uo) <= tol, (name, t, rel(host(u), uo))
        if np.linalg.norm(uto) > 0:
            assert rel(host(ut), uto) <= tol, (name, t, rel(host(ut), uto))
        else:
            assert float(ut.abs().max()) == 0.0, name
    # u alone (ut = NULL) is the same field
    u2 = g.zeros()
    wt.initial_data(g, kind, params, u2, None, t=times[-1])
    assert bool((u2 == u).all())


def test_gaussians_equal_the_host_workload_field(wt, ctx, O):
    """The device Gaussians (the bench's and the server's initial data) equal the host
    field workloads.gaussian_field that the CPU legs start from."""
    g = wt.Mesh.uniform_hex(ctx, 8, 3, 0.0, 1.0, warp_A=0.05, outer_tag=7)
    o = O.OracleMesh(8, 3, A=0.05, outer_tag=7)
    x, y, z = o.coords()
    c, a, w = wt.workloads.pulses(3, 8, amp=(0.5, 1.0), width=(0.05, 0.15), centre=(0.25, 0.75))
    u = g.zeros()
    wt.initial_data(g, wt.IC_GAUSSIANS, wt.gaussian_params(c, a, w), u)
    assert rel(host(u), wt.workloads.gaussian_field(x, y, z, c, a, w)) <= 1e-12


def test_initial_data_errors(wt, ctx):
    g = wt.Mesh.uniform_hex(ctx, 4, 2)
    u = g.zeros()
    with pytest.raises(wt.WaveToyError):
        wt.initial_data(g, 9, [1.0], u)
    with pytest.raises(wt.WaveToyError):       # two pulses announced, one given
        wt.initial_data(g, wt.IC_GAUSSIANS, [2.0, 0.5, 0.5, 0.5, 1.0, 0.1], u)


@pytest.mark.parametrize("N,M,A,periodic", [(8, (3, 2, 4), 0.05, False), (6, (4, 4, 4), 0.05, True),
                                            (5, (2, 3, 2), 0.0, False)])
def test_min_spacing_matches_oracle(wt, ctx, O, N, M, A, periodic):
    g = wt.Mesh.uniform_hex(ctx, N, M, 0.0, 1.0, warp_A=A, periodic=periodic, outer_tag=0 if periodic else 7)
    o = O.OracleMesh(N, M, A=A, periodic=periodic, outer_tag=0 if periodic else 7)
    assert abs(g.min_spacing() - o.min_spacing()) <= 1e-14 * o.min_spacing()
    # the CFL step of the warped ADM workloads (src/evolve.jl:1209-1213)
    sp = wt.workloads.max_speed(wt.workloads.adm_params(4))
    assert abs(0.2 * g.min_spacing() / sp - 0.2 * o.min_spacing() / sp) <= 1e-14 * o.min_spacing() / sp


@pytest.mark.parametrize("kind,M,p", KINDS)
def test_min_spacing_on_patch_meshes(wt, ctx, O, kind, M, p):
    """Curved multi-patch meshes, where the smallest spacing is not along axis 1 of
    every element (the case _min_node_spacing_3d's comment names)."""
    g = wt.Mesh.patches(ctx, kind, 6, M, p)
    o = oracle_from(O, 6, wt.patch_mesh_arrays(kind, 6, M, p))
    assert abs(g.min_spacing() - o.min_spacing()) <= 1e-14 * o.min_spacing()
