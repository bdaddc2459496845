"""GPU acceptance at the configurations' step counts.

The warped-cube ADM solve of the 16^3 x 8^3 configuration (warp A = 0.05, the
perturbed ADM background, one Gaussian pulse of amplitude 1 and width 0.1,
Sommerfeld outer faces, RK4 at CFL 0.2), reduced to 6^3 elements so that the
Float64 oracle runs 500 steps in seconds:
  * the plain FP64 form agrees with the oracle to <= 1e-12 relative L2 after
    200, 300 and 500 steps;
  * the compensated FP32 form (the default FP32 form) to <= 1e-5;
  * the plain FP32 forms (FP32 CUDA cores, split BF16 x3) are held to the
    bound they reach, 5e-5: their FP32 rounding of Phi is amplified by the
    second derivative in Pi-dot, which is what the compensated form removes;
  * the discrete H-norm energy (wave3d_energy, src/wave3d_curved.jl:268-287)
    does not grow: it stays at or below its initial value (the pulse leaves
    through the Sommerfeld faces) and follows the oracle's to 1e-6.
Served-request shapes (elements per axis 16 and 24, n = 8 and 6, three pulses,
ADM scale 1.0) over 2000 steps: the compensated FP32 form stays within 1e-5 of
the FP64 form, whose agreement with the oracle the first test pins.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
TOL32 = 1e-5
TOL32_PLAIN = 5e-5


def rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def host(t):
    return t.detach().double().cpu().numpy()


def c2_reduced(wt, ctx, O, precision, form=None, M=6, seed=11):
    g = wt.Mesh.warped_uniform_hex(ctx, 8, M, 0.0, 1.0, 0.05, outer_tag=wt.SOMMERFELD_BDRY_TAG,
                                   precision=precision)
    if form is not None:
        g.set_fp32_form(form)
    p = wt.workloads.adm_params(seed)
    coef = wt.sample_background3d(g, wt.BG_ADM_PERTURBED, p)
    ws = wt.make_wave3d_workspace(g)
    c, a, w = wt.workloads.pulses(seed, 1, amp=(1.0, 1.0), width=(0.1, 0.1))
    Phi, Pi = g.zeros(), g.zeros()
    wt.initial_state(ws, wt.IC_GAUSSIANS, wt.gaussian_params(c, a, w), Phi, Pi)
    dt = 0.2 * g.min_spacing() / wt.workloads.max_speed(p)
    return g, coef, ws, Phi, Pi, dt, (c, a, w), p


@pytest.fixture(scope="module")
def oracle_run(wt, ctx, O):
    """The oracle's 500-step run of the reduced configuration, with states and
    energies after 0, 200, 300 and 500 steps."""
    M, seed = 6, 11
    o = O.OracleMesh(8, M, A=0.05, outer_tag=7)
    p = wt.workloads.adm_params(seed)
    co = o.background(2, p)
    x, y, z = o.coords()
    c, a, w = wt.workloads.pulses(seed, 1, amp=(1.0, 1.0), width=(0.1, 0.1))
    P = wt.workloads.gaussian_field(x, y, z, c, a, w)
    Q = np.zeros_like(P)
    dt = 0.2 * o.min_spacing() / wt.workloads.max_speed(p)
    bc = O.make_bc([2] * 6)
    out = {0: (P.copy(), Q.copy(), o.energy(co, P, Q, use_metric=True))}
    done = 0
    for ck in (200, 300, 500):
        P, Q = o.evolve_curved(co, P, Q, dt, ck - done, bc=bc, use_metric=True)
        done = ck
        out[ck] = (P.copy(), Q.copy(), o.energy(co, P, Q, use_metric=True))
    return out, dt


@pytest.mark.parametrize("form", ["f64", "compensated", "cuda", "bf16x3"])
def test_reduced_config_against_oracle_200_300_500_steps(wt, ctx, O, oracle_run, form):
    ref, dt_o = oracle_run
    prec = wt.WT_F64 if form == "f64" else wt.WT_F32
    fmap = {"compensated": wt.FP32_COMPENSATED, "cuda": wt.FP32_CUDA_CORES, "bf16x3": wt.FP32_BF16X3}
    g, coef, ws, Phi, Pi, dt, _, _ = c2_reduced(wt, ctx, O, prec, fmap.get(form))
    assert abs(dt - dt_o) <= 1e-14 * dt_o
    bc = wt.make_bc3d([wt.BC_SOMMERFELD] * 6)
    tol = {"f64": TOL64, "compensated": TOL32}.get(form, TOL32_PLAIN)
    E0 = wt.wave3d_energy(Phi, Pi, coef, ws, metric=True)
    assert abs(E0 - ref[0][2]) <= 1e-7 * ref[0][2]
    done = 0
    for ck in (200, 300, 500):
        wt.step_rk4_curved(Phi, Pi, coef, ws, dt, ck - done, bc3d=bc, metric=True)
        done = ck
        Po, Qo, Eo = ref[ck]
        err = rel(np.concatenate([host(Phi), host(Pi)]), np.concatenate([Po, Qo]))
        assert err <= tol, (form, ck, err)
        E = wt.wave3d_energy(Phi, Pi, coef, ws, metric=True)
        assert E <= E0 * (1 + 1e-9) and Eo <= ref[0][2] * (1 + 1e-9), (form, ck, E, E0, Eo)
        assert abs(E - Eo) <= 1e-6 * ref[0][2], (form, ck, E, Eo)
    assert not ctx.nonfinite()


@pytest.mark.parametrize("n,M", [(8, 16), (6, 24)])
def test_served_shape_2000_steps_compensated_vs_f64(wt, ctx, n, M):
    bc = wt.make_bc3d([wt.BC_SOMMERFELD] * 6)
    seed, scale = 17, 1.0
    out = {}
    for prec in (wt.WT_F64, wt.WT_F32):
        g = wt.Mesh.warped_uniform_hex(ctx, n, M, 0.0, 1.0, 0.05, outer_tag=wt.SOMMERFELD_BDRY_TAG, precision=prec)
        p = wt.workloads.adm_params(seed, scale)
        coef = wt.sample_background3d(g, wt.BG_ADM_PERTURBED, p)
        ws = wt.make_wave3d_workspace(g)
        c, a, w = wt.workloads.pulses(seed, 3, amp=(0.5, 1.0), width=(0.05, 0.15), centre=(0.25, 0.75))
        Phi, Pi = g.zeros(), g.zeros()
        wt.initial_state(ws, wt.IC_GAUSSIANS, wt.gaussian_params(c, a, w), Phi, Pi)
        dt = 0.2 * g.min_spacing() / wt.workloads.max_speed(p)
        E0 = wt.wave3d_energy(Phi, Pi, coef, ws, metric=True)
        wt.step_rk4_curved(Phi, Pi, coef, ws, dt, 2000, bc3d=bc, metric=True)
        E = wt.wave3d_energy(Phi, Pi, coef, ws, metric=True)
        assert E <= E0 * (1 + 1e-9)
        out[prec] = np.concatenate([host(Phi), host(Pi)]), E
    err = rel(out[wt.WT_F32][0], out[wt.WT_F64][0])
    assert err <= TOL32, err
    assert abs(out[wt.WT_F32][1] - out[wt.WT_F64][1]) <= 1e-6 * out[wt.WT_F64][1]
    assert not ctx.nonfinite()
