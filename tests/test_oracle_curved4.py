"""CPU tests of the oracle's scalar wave on a prescribed 4-metric
(wave_curved_rhs_mesh! / wave_curved_rhs_conservative_mesh!,
src/wave_curved_rhs.jl), ported from the reference's test/wave_curved_tests.jl:
Minkowski reductions, constant data on the gauge wave, spectra, H-symmetry and a
bounded leapfrog evolution with the metric re-evaluated every step."""
import numpy as np
import pytest


def op_matrix(o, ginv, gam, h, conservative):
    n = o.nn
    L = np.zeros((n, n))
    z = np.zeros(n)
    for k in range(n):
        e = np.zeros(n)
        e[k] = 1.0
        L[:, k] = o.rhs_curved4(e, z, ginv, gam, h, conservative=conservative)
    return L


def test_constant_annihilated_on_gauge_wave(O):
    o = O.OracleMesh(4, 2, periodic=True)
    phi, phid = np.ones(o.nn), np.zeros(o.nn)
    for t in (0.0, 0.13, 0.25, 0.5):
        ginv, gam = o.curved4_background(1, (0.1, 1.0), t)
        for cons in (False, True):
            assert np.max(np.abs(o.rhs_curved4(phi, phid, ginv, gam, 0.5, conservative=cons))) < 1e-10


def test_minkowski_independent_of_phidot_and_conservative_matches_flat(O):
    rng = np.random.default_rng(20260531)
    o = O.OracleMesh(4, 1, periodic=True)
    ginv, gam = o.curved4_background(0)
    phi = rng.standard_normal(o.nn)
    for cons in (False, True):
        a = o.rhs_curved4(phi, rng.standard_normal(o.nn), ginv, gam, 1.0, conservative=cons)
        b = o.rhs_curved4(phi, rng.standard_normal(o.nn), ginv, gam, 1.0, conservative=cons)
        assert np.array_equal(a, b)
    # conservative variant on Minkowski = the flat conservative Laplacian
    a = o.rhs_curved4(phi, np.zeros(o.nn), ginv, gam, 1.0, conservative=True)
    assert np.max(np.abs(a - o.lap_strong_cons(phi, 1.0))) < 1e-12
    o2 = O.OracleMesh(4, 2, periodic=True)
    g2, G2 = o2.curved4_background(0)
    phi2 = rng.standard_normal(o2.nn)
    a2 = o2.rhs_curved4(phi2, np.zeros(o2.nn), g2, G2, 0.5, conservative=True)
    assert np.max(np.abs(a2 - o2.lap_strong_cons(phi2, 0.5))) < 1e-10


def test_minkowski_spectra(O):
    o = O.OracleMesh(3, 2, periodic=True)
    ginv, gam = o.curved4_background(0)
    lam = np.linalg.eigvals(op_matrix(o, ginv, gam, 0.5, False))   # centred flux
    assert lam.real.max() < 0.1 and np.abs(lam.imag).max() < 0.1 and lam.real.min() < -1.0
    L = op_matrix(o, ginv, gam, 0.5, True)                           # conservative
    lam = np.linalg.eigvals(L)
    assert lam.real.max() < 1e-10 and np.abs(lam.imag).max() < 1e-10 and lam.real.min() < -1.0
    x, H, _ = O.gll_ops(3)
    Hn = np.einsum("i,j,k->kji", H, H, H).ravel() * 0.5 ** 3
    Hv = np.tile(Hn, o.Ne)
    HL = Hv[:, None] * L
    assert np.max(np.abs(HL - HL.T)) / np.max(np.abs(HL)) < 1e-12


@pytest.mark.parametrize("cons", [False, True])
def test_leapfrog_on_gauge_wave_bounded(O, cons):
    o = O.OracleMesh(4, 2, periodic=True)
    phi, phid = np.ones(o.nn), np.zeros(o.nn)
    dt, nsteps = 0.01, 300
    ginv, gam = o.curved4_background(1, (0.05, 1.0), 0.0)
    phid += 0.5 * dt * o.rhs_curved4(phi, phid, ginv, gam, 0.5, conservative=cons)
    bound, t = np.max(np.abs(phi - 1)), 0.0
    for _ in range(nsteps):
        phi += dt * phid
        t += dt
        ginv, gam = o.curved4_background(1, (0.05, 1.0), t)
        phid += dt * o.rhs_curved4(phi, phid, ginv, gam, 0.5, conservative=cons)
        bound = max(bound, np.max(np.abs(phi - 1)))
    assert np.all(np.isfinite(phi)) and bound < 0.1


def test_conservative_and_centred_flux_differ_on_gauge_wave(O):
    """test/wave_curved_tests.jl:354-375: on the gauge wave (A = 0.1, d = 1; N = 4, periodic
    2x2x2) the conservative (Mattsson-Nordstrom) and centred-flux forms give different but
    comparable RHS on random data (relative difference between 1e-6 and 10)."""
    o = O.OracleMesh(4, 2, periodic=True)
    ginv, gam = o.curved4_background(1, (0.1, 1.0), 0.0)
    rng = np.random.default_rng(20260601)
    phi, phid = rng.standard_normal(o.nn), rng.standard_normal(o.nn)
    cf = o.rhs_curved4(phi, phid, ginv, gam, 0.5, conservative=False)
    cons = o.rhs_curved4(phi, phid, ginv, gam, 0.5, conservative=True)
    rel = np.max(np.abs(cons - cf)) / np.max(np.abs(cf))
    assert 1e-6 < rel < 10.0
