"""CPU tests of the oracle's time-dependent (spacetime-metric) backgrounds,
MetricBackground3D with SpacetimeMetrics' GaugeWave / SineShift
(src/wave3d_curved.jl:56-71): the oracle's general 3+1 split of the 4-metric
gives the ADM variables the reference states for them (src/evolve.jl:171-195),
and RK4 with the background re-sampled at every stage time converges to the
exact plane-wave solutions the reference gives (Phi = sin(k0 psi))."""
import numpy as np
import pytest


def exact(kind, A, d, k0, t, x):
    k = 2 * np.pi / d
    if kind == 4:  # gauge wave
        C = A * d / (4 * np.pi)
        psi = x - t + 2 * C * np.cos(k * (x - t))
        return np.sin(k0 * psi), -k0 * (1 - A * np.sin(k * (x - t))) * np.cos(k0 * psi)
    C = A * d / (2 * np.pi)   # sine shift
    psi = x + C * np.sin(k * (x - t)) - t
    return np.sin(k0 * psi), -k0 * (1 + A * np.cos(k * (x - t))) * np.cos(k0 * psi)


@pytest.mark.parametrize("kind", [4, 5])
def test_adm_split_matches_stated_variables(O, kind):
    o = O.OracleMesh(4, 2, periodic=True)
    A, d, t = 0.3, 1.0, 0.37
    c = o.background(kind, [A, d, t]).reshape(11, -1)
    x, _, _ = o.coords()
    ph = 2 * np.pi * (x - t) / d
    if kind == 4:
        H = 1 - A * np.sin(ph)
        want = {0: np.sqrt(H), 1: np.sqrt(H), 2: 0 * x, 5: 1 / H}
    else:
        ac = A * np.cos(ph)
        want = {0: 1 + 0 * x, 1: 1 + ac, 2: -ac / (1 + ac), 5: 1 / (1 + ac) ** 2}
    for f, v in want.items():
        assert np.max(np.abs(c[f] - v)) < 1e-14, f
    assert np.max(np.abs(c[[3, 4, 6, 7, 9]])) < 1e-15          # no y, z shift, no off-diagonal metric
    assert np.max(np.abs(c[8] - 1)) < 1e-15 and np.max(np.abs(c[10] - 1)) < 1e-15


@pytest.mark.parametrize("kind", [4, 5])
def test_plane_wave_converges(O, kind):
    """Periodic unit cube, one wavelength along x; error at t = 0.15 drops by more than
    30x when the elements are halved (n = 6: fifth order or better)."""
    A, d, k0, t1 = 0.1, 1.0, 2 * np.pi, 0.15
    speed = 1.0 if kind == 4 else (1 + A) / (1 - A)
    errs = []
    for M in (2, 4):
        o = O.OracleMesh(6, M, periodic=True)
        x, _, _ = o.coords()
        P0, Q0 = exact(kind, A, d, k0, 0.0, x)
        nst = int(np.ceil(t1 / (0.25 * o.min_spacing() / speed)))
        dt = t1 / nst
        P, Q = o.evolve_curved_td(kind, (A, d), 0.0, P0, Q0, dt, nst)
        Pe, Qe = exact(kind, A, d, k0, t1, x)
        errs.append(np.sqrt(np.mean((P - Pe) ** 2)))
    assert errs[1] < 1e-3 and errs[0] / errs[1] > 30, errs
