"""GPU: the bounds-check build (libwavetoy_b200_bc.so, built by
`python wavetoysecondorder.jl_b200/build.py --bounds-check`, -DWT_BOUNDS_CHECK).

compute-sanitizer is closed on this pool, so the debug build checks every index
a kernel reads from the mesh's face-source, neighbour and boundary-slot tables
against the table's range before using it.  A child process loads the debug
library (WAVETOY_B200_LIB) and runs the kernel families on small cases: the
n = 8 FP64 step (fused and two-kernel stages), the compensated and split-BF16
FP32 forms, the generic n = 4, 6 kernels with Dirichlet faces, a batch through
the pipelined kernels, a multi-patch mesh with turned faces, the SIPG RHS and
Kreiss-Oliger dissipation.  It checks that no check fired, and the parent checks
that the results equal the normal library's bit for bit.  Then the child plants
an out-of-range face source and boundary slot (wt_mesh_debug_set_table): the
check reports each, every access stays inside its buffer (the value becomes "no
neighbour" / slot 0) and the context keeps working.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_BC = os.path.join(ROOT, "wavetoysecondorder.jl_b200", "libwavetoy_b200_bc.so")


def _host(t):
    return t.double().cpu().numpy()


def _adm_solve(wt, ctx, N, M, prec=0, form=None, seed=1):
    g = wt.Mesh.uniform_hex(ctx, N, M, outer_tag=7, warp_A=0.05, precision=prec)
    if form is not None:
        g.set_fp32_form(form)
    p = wt.workloads.adm_params(seed)
    c = wt.sample_background3d(g, wt.BG_ADM_PERTURBED, p)
    ws = wt.make_wave3d_workspace(g)
    P, Q = g.zeros(), g.zeros()
    wt.initial_state(ws, wt.IC_GAUSSIANS, wt.gaussian_params(*wt.workloads.pulses(seed, 2)), P, Q)
    dt = 0.2 * g.min_spacing() / wt.workloads.max_speed(p)
    return g, c, ws, P, Q, dt


def _bc(wt, g=None, kind=2):
    """Sommerfeld faces, or Dirichlet / full-Dirichlet faces with seeded boundary data on g."""
    import torch
    if kind == 2:
        return wt.make_bc3d([wt.BC_SOMMERFELD] * 6)
    rng = np.random.default_rng(40 + kind)
    data = [torch.tensor(rng.standard_normal(g.nn), device="cuda").to(g.dtype) for _ in range(5)]
    return wt.make_bc3d([kind] * 6, gPhi=data[0], gPi=data[1], gDx=data[2], gDy=data[3], gDz=data[4])


def case_results(wt, ctx, check):
    """Run every kernel family on a small case; check() after each.  {name: host array}."""
    import torch
    out = {}
    # n = 8 FP64: fused stage kernel, then the two-kernel stages
    for fused in (True, False):
        g, c, ws, P, Q, dt = _adm_solve(wt, ctx, 8, 2)
        ws.set_fused(fused)
        wt.step_rk4_curved(P, Q, c, ws, dt, 3, bc3d=_bc(wt), metric=True)
        out[f"n8_f64_fused{int(fused)}"] = np.concatenate([_host(P), _host(Q)])
        check(f"n8_f64_fused{int(fused)}")
    # n = 8 FP32: compensated (default) and split-BF16 tensor cores; CUDA-core FP32
    for form in (wt.FP32_COMPENSATED, wt.FP32_BF16X3, wt.FP32_CUDA_CORES):
        g, c, ws, P, Q, dt = _adm_solve(wt, ctx, 8, 2, prec=1, form=form)
        wt.step_rk4_curved(P, Q, c, ws, dt, 3, bc3d=_bc(wt), metric=True)
        out[f"n8_f32_form{form}"] = np.concatenate([_host(P), _host(Q)])
        check(f"n8_f32_form{form}")
    # generic kernels (n = 4, 6) and n = 8 with Dirichlet (FP64 data), Sommerfeld and full-Dirichlet faces
    for N, prec, kind in ((4, 0, 1), (6, 0, 2), (6, 1, 2), (8, 0, 4)):
        g, c, ws, P, Q, dt = _adm_solve(wt, ctx, N, 3, prec=prec, seed=N)
        wt.step_rk4_curved(P, Q, c, ws, dt, 3, bc3d=_bc(wt, g, kind), metric=True)
        out[f"bc_n{N}_p{prec}_k{kind}"] = np.concatenate([_host(P), _host(Q)])
        check(f"bc_n{N}_p{prec}_k{kind}")
    # a batch: n = 4 and 6 through the pipelined kernels, n = 8 through the work-list kernels
    solves = [_adm_solve(wt, ctx, N, 2, seed=10 + N) for N in (4, 6, 8)]
    b = wt.Batch(ctx, autotune=False)
    b.set_variant(2, 2)
    for g, c, ws, P, Q, dt in solves:
        b.add(P, Q, c, ws, dt, _bc(wt))
    b.step(4)
    for (g, c, ws, P, Q, dt), N in zip(solves, (4, 6, 8)):
        out[f"batch_n{N}"] = np.concatenate([_host(P), _host(Q)])
    check("batch")
    # a multi-patch mesh (turned faces): the RHS
    g = wt.Mesh.patches(ctx, wt.MESH_CUBED_CUBE, 5, 2, (0.3,))
    c = wt.sample_background3d(g, wt.BG_ADM_PERTURBED, wt.workloads.adm_params(3))
    ws = wt.make_wave3d_workspace(g)
    rng = np.random.default_rng(5)
    P = torch.tensor(rng.standard_normal(g.nn), device="cuda")
    Q = torch.tensor(rng.standard_normal(g.nn), device="cuda")
    Pd, Qd = g.zeros(), g.zeros()
    wt.wave3d_curved_rhs(Pd, Qd, P, Q, c, ws, eps_KO=0.0, bc3d=_bc(wt), metric=True)
    out["patches_rhs"] = np.concatenate([_host(Pd), _host(Qd)])
    check("patches_rhs")
    # Kreiss-Oliger dissipation (line kernels and apply_D) on a warped mesh
    g, c, ws, P, Q, dt = _adm_solve(wt, ctx, 6, 3, seed=6)
    Pd, Qd = g.zeros(), g.zeros()
    wt.wave3d_curved_rhs(Pd, Qd, P, Q, c, ws, eps_KO=0.1, bc3d=_bc(wt), metric=True)
    out["ko_rhs"] = np.concatenate([_host(Pd), _host(Qd)])
    check("ko_rhs")
    # the SIPG RHS with Sommerfeld faces
    g = wt.Mesh.uniform_hex(ctx, 6, 3, outer_tag=7)
    ws = wt.make_wave3d_workspace(g)
    u = torch.tensor(rng.standard_normal(g.nn), device="cuda")
    ut = torch.tensor(rng.standard_normal(g.nn), device="cuda")
    utt = g.zeros()
    wt.rhs_wave3d(utt, u, ut, [0.1, -0.2, 0.3, 0.0, 0.5, -0.4], ws, tau=20.0, sommerfeld_R=1.5)
    out["sipg_rhs"] = _host(utt)
    check("sipg_rhs")
    return out


def planted_words(wt, ctx):
    """Plant an out-of-range face source, then boundary slot, in an n = 6 and an n = 8 mesh
    and step; {name: bounds word or finiteness}."""
    import torch
    words = {}
    for N in (6, 8):
        for table, value, name in ((wt.TABLE_FACE_SOURCE, None, "src"), (wt.TABLE_BOUNDARY_SLOT, 1 << 20, "slot")):
            g, c, ws, P, Q, dt = _adm_solve(wt, ctx, N, 3, seed=N)
            if value is None:
                value = 64 * (g.Ne + 1000)   # element 0's +x face: a neighbour past the last element
            wt.debug_set_table(g, table, 0, 1 if name == "src" else 0, value)  # face 0 of element 0 is outer
            wt.step_rk4_curved(P, Q, c, ws, dt, 2, bc3d=_bc(wt), metric=True)
            words[f"{name}_n{N}"] = ctx.bounds_status()
            words[f"{name}_n{N}_finite"] = int(bool(torch.isfinite(P).all() and torch.isfinite(Q).all()))
    g, c, ws, P, Q, dt = _adm_solve(wt, ctx, 8, 2)
    wt.step_rk4_curved(P, Q, c, ws, dt, 2, bc3d=_bc(wt), metric=True)
    words["clean_after"] = ctx.bounds_status()
    return words


def _child(out_path):
    """Entry of the child process: WAVETOY_B200_LIB names the bounds-check library."""
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    from conftest import load_package
    wt = load_package()
    assert wt.LIB_PATH == LIB_BC and wt.build_flags() & wt.BUILD_BOUNDS_CHECK
    ctx = wt.Context(0)
    fired = []

    def check(name):
        w = ctx.bounds_status()
        if w:
            fired.append(f"{name}:{w}")

    res = case_results(wt, ctx, check)
    words = planted_words(wt, ctx)
    assert not ctx.nonfinite()
    np.savez(out_path, **res, **{"w_" + k: np.array(v) for k, v in words.items()},
             fired=np.array(";".join(fired)))


@pytest.fixture(scope="module")
def debug_run(tmp_path_factory):
    if not os.path.exists(LIB_BC):
        pytest.skip("libwavetoy_b200_bc.so is not built (build.py --bounds-check)")
    out = str(tmp_path_factory.mktemp("bounds") / "bc.npz")
    env = dict(os.environ, WAVETOY_B200_LIB=LIB_BC)
    r = subprocess.run([sys.executable, os.path.abspath(__file__), out], env=env, capture_output=True, text=True,
                       timeout=900)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-4000:]
    return dict(np.load(out))


def test_no_check_fires_and_results_equal_normal_build(wt, ctx, debug_run):
    assert str(debug_run["fired"]) == ""
    ref = case_results(wt, ctx, lambda name: None)
    assert set(ref) == {k for k in debug_run if not k.startswith("w_") and k != "fired"}
    for k, v in ref.items():
        assert np.array_equal(v, debug_run[k]), k


def test_planted_out_of_range_entries_are_reported(debug_run):
    for N in (6, 8):
        assert int(debug_run[f"w_src_n{N}"]) == 1, N      # bit 0: an element index
        assert int(debug_run[f"w_slot_n{N}"]) == 2, N     # bit 1: a boundary slot
        assert int(debug_run[f"w_src_n{N}_finite"]) == 1 and int(debug_run[f"w_slot_n{N}_finite"]) == 1
    assert int(debug_run["w_clean_after"]) == 0


def test_normal_build_has_no_checks(wt, ctx):
    if wt.LIB_PATH == LIB_BC:
        pytest.skip("the whole suite runs under the bounds-check library")
    assert not wt.build_flags() & wt.BUILD_BOUNDS_CHECK
    assert wt.build_flags() & wt.BUILD_NVTX
    assert ctx.bounds_status() == 0
    g = wt.Mesh.uniform_hex(ctx, 4, 2)
    with pytest.raises(wt.WaveToyError) as ei:
        wt.debug_set_table(g, wt.TABLE_FACE_SOURCE, 0, 1, -1)
    assert ei.value.code == -4


if __name__ == "__main__":
    _child(sys.argv[1])
