"""Property tests of the CPU oracle, ported from the reference's 3D test suite.

The reference ships no golden vectors; its tests pin the discretisation by
properties (spectrum, free-stream, convergence, energy, symmetry).  These ports
are the acceptance gate that the oracle's restatement of the unvendored
HexSBPSAT/HexMeshes arithmetic is the reference's scheme class.  Each test
cites the reference test it follows.
"""
import math

import numpy as np
import pytest


def dense(f, n):
    A = np.zeros((n, n))
    for j in range(n):
        e = np.zeros(n)
        e[j] = 1.0
        A[:, j] = f(e)
    return A


@pytest.mark.parametrize("N", [2, 3, 4, 5, 6, 7, 8])
def test_gll_sbp_identity(O, N):
    """H G + (H G)^T = B with B = diag(-1,0,...,0,1) (README.md:14-19)."""
    x, H, G = O.gll_ops(N)
    Q = np.diag(H) @ G
    B = np.zeros((N, N)); B[0, 0] = -1; B[-1, -1] = 1
    assert np.abs(Q + Q.T - B).max() < 1e-13
    assert abs(H.sum() - 1.0) < 1e-14
    assert x[0] == 0.0 and x[-1] == 1.0


def test_apply_D_exactly_skew_on_affine(O):
    """H*D + (H*D)^T = 0 for apply_D! on an affine periodic mesh (METHODS.md:256-264)."""
    m = O.OracleMesh(4, 2, periodic=True)
    Hp = m.get("Hphys")
    for d in range(3):
        HA = np.diag(Hp) @ dense(lambda v: m.apply_D(v, d), m.nn)
        assert np.abs(HA + HA.T).max() < 1e-14


def test_metric_identity_and_free_stream(O):
    """Curl-form metric terms: sum_al Dhat_al(J a^al_i) = 0 to <= 1e-10, grad/div of a
    constant vanish (METHODS.md:158-166; test/wave3d_tests.jl:109-125 asserts <= 1e-9)."""
    m = O.OracleMesh(4, 3, A=0.05, outer_tag=7)
    c = np.full(m.nn, 2.5)
    g = m.grad3d(c)
    assert max(np.abs(v).max() for v in g) <= 1e-9
    assert np.abs(m.div3d(c, -0.3 * c, 0.7 * c)).max() <= 1e-9
    coef = m.background(0)
    bc = O.make_bc([O.BC_SOMMERFELD] * 6)
    Pd, Qd = m.rhs_curved(coef, c, np.zeros(m.nn), eps_ko=0.0, bc=bc, use_metric=True)
    assert np.abs(Pd).max() <= 1e-9 and np.abs(Qd).max() <= 1e-9


def test_split_form_pair_is_skew_adjoint(O):
    """Hd*grad and Hd*div are adjoint with opposite sign on a periodic warped mesh
    (skew-adjoint split form, METHODS.md:124-135)."""
    m = O.OracleMesh(3, 2, A=0.05, periodic=True)
    Hd = m.get("Hd")
    rng = np.random.default_rng(7)
    u = rng.standard_normal(m.nn)
    F = [rng.standard_normal(m.nn) for _ in range(3)]
    g = m.grad3d(u)
    dv = m.div3d(*F)
    lhs = sum((Hd * g[i] * F[i]).sum() for i in range(3)) + (Hd * u * dv).sum()
    assert abs(lhs) < 1e-12


@pytest.mark.parametrize("periodic", [True, False])
def test_rhs_spectrum_affine(O, periodic):
    """max Re(lambda) <= 1e-5 max|lambda|, N=4, M=2, eps_KO=0.1, periodic and
    Sommerfeld (test/wave3d_tests.jl:71-89)."""
    m = O.OracleMesh(4, 2, periodic=periodic, outer_tag=7)
    coef = m.background(0)
    bc = None if periodic else O.make_bc([O.BC_SOMMERFELD] * 6)
    nn = m.nn
    A = dense(lambda x: np.concatenate(m.rhs_curved(coef, x[:nn].copy(), x[nn:].copy(), eps_ko=0.1, bc=bc)), 2 * nn)
    lam = np.linalg.eigvals(A)
    assert lam.real.max() <= 1e-5 * np.abs(lam).max()


def test_rhs_spectrum_curvilinear_sommerfeld(O):
    """Curved Sommerfeld spectrum stable (test/wave3d_tests.jl:126-141, there on the
    cubed cube; here on the warped cube, eps_KO = 0.1)."""
    m = O.OracleMesh(4, 2, A=0.05, outer_tag=7)
    coef = m.background(0)
    bc = O.make_bc([O.BC_SOMMERFELD] * 6)
    nn = m.nn
    A = dense(lambda x: np.concatenate(m.rhs_curved(coef, x[:nn].copy(), x[nn:].copy(), eps_ko=0.1, bc=bc,
                                                    use_metric=True)), 2 * nn)
    lam = np.linalg.eigvals(A)
    assert lam.real.max() <= 1e-5 * np.abs(lam).max()


def test_rhs_spectrum_adm_background(O):
    """Warped mesh + perturbed ADM background (the warped-cube workload's class) with
    Sommerfeld faces: max Re(lambda) at round-off."""
    import conftest
    wt = conftest.load_package()
    m = O.OracleMesh(4, 2, A=0.05, outer_tag=7)
    coef = m.background(2, wt.workloads.adm_params(2))
    bc = O.make_bc([O.BC_SOMMERFELD] * 6)
    nn = m.nn
    A = dense(lambda x: np.concatenate(m.rhs_curved(coef, x[:nn].copy(), x[nn:].copy(), eps_ko=0.0, bc=bc,
                                                    use_metric=True)), 2 * nn)
    lam = np.linalg.eigvals(A)
    assert lam.real.max() <= 1e-5 * np.abs(lam).max()


def test_periodic_plane_wave_energy_and_convergence(O):
    """Periodic plane wave, N=4: energy drift < 1e-3, error ratio M=4 -> 8 > 4
    (test/wave3d_tests.jl:50-69)."""
    kap = 2 * math.pi
    om = kap * math.sqrt(3.0)
    errs = []
    for M in (4, 8):
        m = O.OracleMesh(4, M, periodic=True)
        coef = m.background(0)
        x, y, z = m.coords()
        Phi = np.sin(kap * (x + y + z))
        Pi = -om * np.cos(kap * (x + y + z))
        xg, _, _ = O.gll_ops(4)
        dxmin = np.diff(xg).min() / M
        dt = 0.1 * dxmin
        nst = math.ceil(0.2 / dt)
        E0 = m.energy(coef, Phi, Pi)
        P1, Q1 = m.evolve_curved(coef, Phi, Pi, dt, nst)
        E1 = m.energy(coef, P1, Q1)
        assert abs(E1 / E0 - 1) < 1e-3
        Hp = m.get("Hphys")
        ex = np.sin(kap * (x + y + z) - om * nst * dt)
        errs.append(math.sqrt(((P1 - ex) ** 2 * Hp).sum()))
    assert errs[0] / errs[1] > 4


def test_noise_bounded_sommerfeld_ko(O):
    """sqrt(eps) noise with Sommerfeld + KO stays < 1000 amp over t = 8
    (test/wave3d_tests.jl:91-101; numpy seed stands in for Random.seed!(20260604))."""
    m = O.OracleMesh(4, 2, outer_tag=7)
    coef = m.background(0)
    rng = np.random.default_rng(20260604)
    amp = math.sqrt(np.finfo(float).eps)
    Phi = amp * rng.standard_normal(m.nn)
    Pi = amp * rng.standard_normal(m.nn)
    xg, _, _ = O.gll_ops(4)
    dt = 0.1 * np.diff(xg).min() / 2
    nst = math.ceil(8 / dt)
    P1, _ = m.evolve_curved(coef, Phi, Pi, dt, nst, eps_ko=0.1, bc=O.make_bc([O.BC_SOMMERFELD] * 6))
    assert np.all(np.isfinite(P1)) and np.abs(P1).max() < 1000 * amp


def test_sommerfeld_energy_non_increasing(O):
    """Noise + Sommerfeld + KO: energy never exceeds its initial value by more than
    1e-6 relative (test/evolve3d_tests.jl:30-37, test/evolve3d_curv_tests.jl:36-45)."""
    m = O.OracleMesh(4, 2, A=0.05, outer_tag=7)
    coef = m.background(0)
    rng = np.random.default_rng(1234)
    amp = math.sqrt(np.finfo(float).eps)
    Phi = amp * rng.standard_normal(m.nn)
    Pi = amp * rng.standard_normal(m.nn)
    dt = 0.1 * m.min_spacing() / math.sqrt(3)
    _, _, E = m.evolve_curved(coef, Phi, Pi, dt, 60, eps_ko=0.1, bc=O.make_bc([O.BC_SOMMERFELD] * 6),
                              use_metric=True, record_energy=True)
    assert E.max() <= E[0] * (1 + 1e-6)
    assert E[-1] < E[0]


def _sipg_HL(O, N, M=2):
    m = O.OracleMesh(N, M, outer_tag=0)
    nn = m.nn
    Hp = m.get("Hphys")
    L0 = dense(lambda v: m.rhs_sipg(v, np.zeros(nn), tau=0.0), nn)
    L1 = dense(lambda v: m.rhs_sipg(v, np.zeros(nn), tau=1.0), nn)
    return m, np.diag(Hp) @ L0, np.diag(Hp) @ (L1 - L0)


def test_sipg_symmetric_and_threshold_pins_readme(O):
    """H L_SAT is symmetric; its coercivity threshold at the reference driver's
    default N = 5 reproduces the documented 'tau >~ 17 in unit-element
    coordinates' (README.md:76-80)."""
    m, HL0, HP = _sipg_HL(O, 5)
    for tau in (10.0, 30.0):
        HL = HL0 + tau * HP
        assert np.abs(HL - HL.T).max() <= 1e-12 * np.abs(HL).max()
    lo, hi = 1.0, 60.0
    for _ in range(30):
        mid = 0.5 * (lo + hi)
        if np.linalg.eigvalsh(0.5 * (HL0 + mid * HP + (HL0 + mid * HP).T)).max() < 0:
            hi = mid
        else:
            lo = mid
    assert 15.0 < hi < 18.0, hi


def test_sipg_tau_threshold_n6_is_above_20(O):
    """At n = 6 the coercivity threshold exceeds tau = 20: H L_SAT has a positive
    eigenvalue at tau = 20 and none at 1.5 (N-1)^2 = 37.5 (the reference driver's
    choice, src/evolve.jl:964-970)."""
    m, HL0, HP = _sipg_HL(O, 6)
    assert np.linalg.eigvalsh(0.5 * (HL0 + 20 * HP + (HL0 + 20 * HP).T)).max() > 0
    assert np.linalg.eigvalsh(0.5 * (HL0 + 37.5 * HP + (HL0 + 37.5 * HP).T)).max() < 0


def test_sipg_analytic_evolution(O):
    """u = sin(2 pi x) sin(2 pi y) sin(2 pi z) cos(omega t), Dirichlet cube, N=4, M=4,
    tau = 1.5 (N-1)^2, dt = 0.5 dx / sqrt(3), t = 1/2: max error < 1e-2
    (test/kernels3d_tests.jl:61-105; RK4 here in place of KahanLi8)."""
    N, M = 4, 4
    m = O.OracleMesh(N, M, outer_tag=0)
    x, y, z = m.coords()
    k = 2 * math.pi
    om = math.sqrt(3) * k
    u0 = np.sin(k * x) * np.sin(k * y) * np.sin(k * z)
    xg, _, _ = O.gll_ops(N)
    dx = np.diff(xg).min() / M
    dt = 0.5 * dx / math.sqrt(3)
    nst = int(round(0.5 / dt))
    dt = 0.5 / nst
    u, v = m.evolve_sipg(u0, np.zeros_like(u0), dt, nst, tau=1.5 * (N - 1) ** 2)
    assert np.abs(u - u0 * math.cos(om * 0.5)).max() < 1e-2


def test_strong_uniform_periodic_regression(O):
    """wave_strong_rhs_mesh! equals wave_lap_strong_conservative_mesh! on the
    uniform periodic cube to 1e-10 (test/wave_strong_rhs_tests.jl:54-70)."""
    m = O.OracleMesh(4, 2, periodic=True)
    rng = np.random.default_rng(20260601)
    u = rng.standard_normal(m.nn)
    ut = rng.standard_normal(m.nn)
    assert np.abs(m.rhs_strong(u, ut) - m.lap_strong_cons(u, 0.5)).max() < 1e-10


def test_strong_warped_A0_equals_flat(O):
    """Warped builder at A = 0 reproduces the flat path (test/dirichlet_warped_tests.jl:19-36)."""
    m0 = O.OracleMesh(4, 3, outer_tag=0)
    m1 = O.OracleMesh(4, 3, A=0.0, outer_tag=0)
    rng = np.random.default_rng(20260605)
    u = rng.standard_normal(m0.nn)
    ut = rng.standard_normal(m0.nn)
    assert np.abs(m0.rhs_strong(u, ut) - m1.rhs_strong(u, ut)).max() < 1e-10


def _rayleigh(O, M, A=0.0, N=4, k=math.pi, periodic=False):
    m = O.OracleMesh(N, M, A=A, periodic=periodic, outer_tag=0)
    x, y, z = m.coords()
    u = np.sin(k * x) * np.sin(k * y) * np.sin(k * z)
    Hp = m.get("Hphys")
    utt = m.rhs_strong(u, np.zeros_like(u))
    return -np.dot(u, Hp * utt) / np.dot(u, Hp * u)


def test_strong_dirichlet_rayleigh(O):
    """Rayleigh quotient -> 3 pi^2 to < 1e-3 at M=4, and h-refinement ratios > 4
    (test/dirichlet_cube_tests.jl:58-108)."""
    lam = 3 * math.pi ** 2
    errs = [abs(_rayleigh(O, M) - lam) for M in (2, 4, 8)]
    assert errs[1] / lam < 1e-3
    assert errs[1] < errs[0] / 4 and errs[2] < errs[1] / 4 and errs[2] < 1e-3


def test_strong_warped_dirichlet_rayleigh(O):
    """Warped A = 0.05: Rayleigh quotient within 5% at M=4 and geometric-mean
    convergence > 4 over M = 2, 4, 8 (test/dirichlet_warped_tests.jl:59-78)."""
    lam = 3 * math.pi ** 2
    assert abs(_rayleigh(O, 4, A=0.05) - lam) / lam < 0.05
    errs = [abs(_rayleigh(O, M, A=0.05) - lam) for M in (2, 4, 8)]
    assert (errs[0] / errs[-1]) ** 0.5 > 4 and errs[-1] < 1e-3


def test_strong_periodic_warped_rayleigh(O):
    """The periodic warped cube (test/periodic_warped_tests.jl:56-92): the H_phys-weighted
    Rayleigh quotient of the strong-form RHS on sin(2 pi x) sin(2 pi y) sin(2 pi z) (physical
    coordinates, N = 4) is continuous in the warp A (A = 0 within 0.01 of 3 (2 pi)^2, larger at
    A = 0.1, below 5 there) and converges at A = 0.05 (errors shrink at least 3 and 50 times
    from M = 2 to 4 and 8, ending below 1e-2)."""
    lam = 3 * (2 * np.pi) ** 2

    def ray(A, M):
        o = O.OracleMesh(4, M, A=A, periodic=True, outer_tag=0)
        x, y, z = o.coords()
        u = np.sin(2 * np.pi * x) * np.sin(2 * np.pi * y) * np.sin(2 * np.pi * z)
        H = o.get("Hphys")
        return -np.dot(u, H * o.rhs_strong(u, np.zeros_like(u))) / np.dot(u, H * u)

    errs = [abs(ray(A, 4) - lam) for A in (0.0, 0.01, 0.05, 0.1)]
    assert errs[0] < 0.01 and errs[3] > errs[0] and errs[3] < 5
    errs = [abs(ray(0.05, M) - lam) for M in (2, 4, 8)]
    assert all(e > 0 for e in errs)
    assert errs[1] < errs[0] / 3 and errs[2] < errs[1] / 50 and errs[2] < 1e-2


def test_strong_dirichlet_spectrum_flat(O):
    """Flat Dirichlet cube: spectrum real and negative (test/dirichlet_cube_tests.jl:110-130)."""
    m = O.OracleMesh(3, 2, outer_tag=0)
    L = dense(lambda v: m.rhs_strong(v, np.zeros(m.nn)), m.nn)
    lam = np.linalg.eigvals(L)
    assert lam.real.max() < 1e-10 and np.abs(lam.imag).max() < 1e-10 and lam.real.min() < -1


def test_lap_strong_cons_H_symmetric(O):
    """H_phys * L symmetric and -H L positive semi-definite for the
    Mattsson-Nordstrom form (test/wave_lap_strong_conservative_tests.jl:129-154)."""
    m = O.OracleMesh(3, 2, periodic=True)
    Hp = m.get("Hphys")
    HL = np.diag(Hp) @ dense(lambda v: m.lap_strong_cons(v, 0.5), m.nn)
    assert np.abs(HL - HL.T).max() < 1e-12 * np.abs(HL).max()
    assert np.linalg.eigvalsh(0.5 * (HL + HL.T)).max() < 1e-10


def test_lap_strong_cons_constants_and_rayleigh_convergence(O):
    """The periodic conservative strong Laplacian (test/wave_lap_strong_mesh_tests.jl:45-135):
    a constant is in its kernel, and the H_phys-weighted Rayleigh quotient of
    sin(2 pi x) sin(2 pi y) sin(2 pi z) converges to the eigenvalue 3 (2 pi)^2 at N = 4 with
    error ratios of at least 5, 50 and 10 from M = 1 to 2, 4 and 8, ending below 1e-3."""
    m = O.OracleMesh(3, 2, periodic=True)
    assert np.abs(m.lap_strong_cons(np.ones(m.nn), 0.5)).max() < 1e-12
    lam = 3 * (2 * np.pi) ** 2
    errs = []
    for M in (1, 2, 4, 8):
        m = O.OracleMesh(4, M, periodic=True)
        x, y, z = m.coords()
        u = np.sin(2 * np.pi * x) * np.sin(2 * np.pi * y) * np.sin(2 * np.pi * z)
        Hp = m.get("Hphys")
        errs.append(abs(-np.dot(u, Hp * m.lap_strong_cons(u, 1.0 / M)) / np.dot(u, Hp * u) - lam))
    assert all(e > 0 for e in errs)
    assert errs[1] < errs[0] / 5 and errs[2] < errs[1] / 50 and errs[3] < errs[2] / 10
    assert errs[3] < 1e-3


def test_lap_strong_cons_leapfrog_energy_is_second_order(O):
    """Leapfrog on the periodic 2x2x2, N = 3 conservative strong Laplacian
    (test/wave_lap_strong_mesh_tests.jl:138-189): the discrete energy's oscillation stays
    below 0.5 at dt = 0.5 * 2 / omega_max over 2000 steps and shrinks more than 3 times when
    dt halves (O(dt^2))."""
    m = O.OracleMesh(3, 2, periodic=True)
    L = dense(lambda v: m.lap_strong_cons(v, 0.5), m.nn)
    Hp = m.get("Hphys")
    w_max = np.sqrt(-np.linalg.eigvals(L).real.min())
    x, y, z = m.coords()
    u0 = np.sin(2 * np.pi * x) * np.sin(2 * np.pi * y) * np.sin(2 * np.pi * z)

    def energy(u, v):
        return 0.5 * v @ (Hp * v) + 0.5 * u @ (Hp * -(L @ u))

    def envelope(factor, nsteps):
        dt = factor * 2 / w_max
        u = u0.copy()
        Lu = L @ u
        v = 0.5 * dt * Lu
        E0 = energy(u, v - 0.5 * dt * Lu)
        lo = hi = E0
        for _ in range(nsteps):
            u = u + dt * v
            Lu = L @ u
            v = v + dt * Lu
            E = energy(u, v - 0.5 * dt * Lu)
            lo, hi = min(lo, E), max(hi, E)
        assert np.isfinite(E)
        return E0, (hi - lo) / E0

    E0a, env_a = envelope(0.5, 2000)
    _, env_b = envelope(0.25, 4000)
    assert E0a > 0 and env_a < 0.5 and env_b < env_a / 3


def test_classify_face(O):
    """classify_face3d flat => subluminal (test/wave3d_tests.jl:103-107)."""
    import conftest
    wt = conftest.load_package()
    assert wt.classify_face3d(1.0, 0.0, 0.0, 0.0, 1.0, 1.0, 1.0, 1, 1) == wt.FACE_SUBLUMINAL
    assert wt.classify_face3d(1.0, 0.0, 0.0, 0.0, 1.0, 1.0, 1.0, 3, -1) == wt.FACE_SUBLUMINAL
    assert wt.classify_face1d(1.0, 2.0, 1) == wt.FACE_INFLOW
    assert wt.classify_face1d(1.0, 2.0, -1) == wt.FACE_OUTFLOW
    assert wt.classify_face1d(1.0, 1.0, 1) == wt.FACE_SONIC
    with pytest.raises(ValueError):
        wt.validate_bc1d(wt.FACE_OUTFLOW, wt.BC_SOMMERFELD, "-x side")
    with pytest.raises(ValueError):
        wt.bc1d_kind("bogus")


def adm_no_shift(wt, seed, scale=1.0):
    """The perturbed ADM background's parameters with zero shift (beta = 0)."""
    p = list(wt.workloads.adm_params(seed, scale))
    p[1] = 0.0
    return p


def test_lapse_weighted_energy_is_conserved_without_shift(O, wt):
    """The reference's wave3d_energy is exactly conserved only for alpha = 1
    (src/wave3d_curved.jl:263-266).  With a static lapse alpha != 1 and zero shift,
    the semi-discrete split-form system conserves the alpha-weighted norm
    E_a = 1/2 sum [(alpha/sqrtg) Pi^2 + alpha sqrtg gu^{ij} dPhi_i dPhi_j] Hd (the
    gradient/divergence pair is skew-adjoint in Hd): dE_a/dt = 0 to round-off on a
    periodic warped mesh, while d/dt of the reference energy is not."""
    N, M = 5, 2
    m = O.OracleMesh(N, M, A=0.05, periodic=True)
    coef = m.background(2, adm_no_shift(wt, 7, 2.0))
    nn = m.nn
    rng = np.random.default_rng(3)
    x, y, z = m.coords()
    Phi = np.sin(2 * np.pi * x) * np.cos(2 * np.pi * y) + 0.3 * np.sin(2 * np.pi * (y + z))
    Pi = 0.5 * np.cos(2 * np.pi * (x - z)) + 0.1 * rng.standard_normal(nn)
    Phid, Pid, D = m.rhs_curved(coef, Phi, Pi, eps_ko=0.0, use_metric=True, want_grad=True)
    _, _, Dd = m.rhs_curved(coef, Phid, Pi, eps_ko=0.0, use_metric=True, want_grad=True)
    Hd = m.get("Hd")
    al, sg = coef[:nn], coef[nn:2 * nn]
    gu = [coef[(5 + c) * nn:(6 + c) * nn] for c in range(6)]   # g11 g12 g13 g22 g23 g33
    K = np.array([[gu[0], gu[1], gu[2]], [gu[1], gu[3], gu[4]], [gu[2], gu[4], gu[5]]])
    g = D.reshape(3, nn)
    gd = Dd.reshape(3, nn)
    Kg = np.einsum("ijn,jn->in", K, g)

    def rate(w):  # d/dt of 1/2 sum w [Pi^2/sqrtg + sqrtg g.gu.g] Hd along the RHS
        return np.sum(Hd * w * (Pi * Pid / sg + sg * np.sum(gd * Kg, axis=0)))

    scale = np.sum(Hd * al * (np.abs(Pi * Pid) / sg + sg * np.abs(np.sum(gd * Kg, axis=0))))
    assert abs(rate(al)) < 1e-12 * scale
    assert abs(rate(np.ones(nn))) > 1e-6 * scale
    # the oracle's weighted energy is that norm
    Ea = 0.5 * np.sum(Hd * al * (Pi ** 2 / sg + sg * np.sum(g * Kg, axis=0)))
    assert abs(m.energy(coef, Phi, Pi, use_metric=True, lapse=True) - Ea) < 1e-13 * Ea


@pytest.mark.parametrize("N", [4, 5])
def test_sommerfeld_faces_absorb_an_outgoing_pulse(O, N):
    """The reference's absorption checks (test/sommerfeld_tests.jl:132-176: an outgoing pulse
    loses >= 95 % of its SIPG energy through Sommerfeld faces by t = 1.5, tau = 1.5 (N-1)^2,
    and BGT-1 leaves a smaller residual than BGT-0), on the unit cube, where this SIPG path
    runs (the reference runs them on the inflated cube).  With Dirichlet faces instead, the
    energy stays (the pulse is reflected)."""
    tau = 1.5 * (N - 1) ** 2
    ratio = {}
    for tag in (7, 1):
        o = O.OracleMesh(N, 4, A=0.0, outer_tag=tag)
        x, y, z = o.coords()
        u, v = O.ic_outgoing_pulse(x, y, z, 0.0, 1.0, 0.2, 0.07, 0.5, 0.5, 0.5)
        dt = 0.2 * o.min_spacing()
        ue, ve = o.evolve_sipg(u, v, dt, int(np.ceil(1.5 / dt)), tau=tau)
        assert np.all(np.isfinite(ue))
        if tag == 7:
            assert np.abs(ue).max() < 1.0                # no blow-up; the initial peak is about 5.3
        ratio[tag] = o.energy_sipg(ue, ve, tau) / o.energy_sipg(u, v, tau)
    assert ratio[7] < 0.05
    assert ratio[1] > 0.95
    # T3 (test/sommerfeld_tests.jl:155-176): BGT-1's +u/R term (R = 0.5, the faces' distance
    # from the pulse centre) leaves under 0.7 of BGT-0's largest residual value
    o = O.OracleMesh(N, 4, A=0.0, outer_tag=7)
    x, y, z = o.coords()
    u, v = O.ic_outgoing_pulse(x, y, z, 0.0, 1.0, 0.2, 0.07, 0.5, 0.5, 0.5)
    dt = 0.2 * o.min_spacing()
    mx = {R: np.abs(o.evolve_sipg(u, v, dt, int(np.ceil(1.5 / dt)), tau=tau, R=R)[0]).max() for R in (np.inf, 0.5)}
    assert mx[0.5] < 0.7 * mx[np.inf]
