"""Fixed-step explicit Runge-Kutta methods of pick_integrator_first_order
(src/evolve.jl:43-48, run with adaptive = false): the library's Tsit5 tableau
(wt_erk_tableau, host only) is the oracle's and satisfies every order condition
up to order 5; the oracle's fixed-step Tsit5 converges at fifth order in time
(RK4 at fourth) on a semi-discrete curvilinear problem, with a static and with
a time-dependent background."""
import numpy as np
import pytest


def order_conditions(c, A, b):
    """Residuals of the 17 order conditions of orders 1-5 (the elementary weights of
    the rooted trees with at most 5 vertices)."""
    e = np.ones_like(c)
    Ac, Ac2, Ac3 = A @ c, A @ c ** 2, A @ c ** 3
    AAc, AAc2, AcAc = A @ Ac, A @ Ac2, A @ (c * Ac)
    return [b @ e - 1, b @ c - 1 / 2, b @ c ** 2 - 1 / 3, b @ Ac - 1 / 6, b @ c ** 3 - 1 / 4, b @ (c * Ac) - 1 / 8,
            b @ Ac2 - 1 / 12, b @ AAc - 1 / 24, b @ c ** 4 - 1 / 5, b @ (c ** 2 * Ac) - 1 / 10,
            b @ (c * Ac2) - 1 / 15, b @ (c * AAc) - 1 / 30, b @ Ac ** 2 - 1 / 20, b @ Ac3 - 1 / 20,
            b @ AcAc - 1 / 40, b @ AAc2 - 1 / 60, b @ (A @ AAc) - 1 / 120]


def test_tsit5_tableau(wt, O):
    c, A, b = wt.erk_tableau(wt.ERK_TSIT5)
    co, Ao, bo = O.erk_tableau(1)
    assert np.array_equal(c, co) and np.array_equal(A, Ao) and np.array_equal(b, bo)
    assert np.allclose(A.sum(1), c, atol=1e-15, rtol=0)
    assert max(abs(r) for r in order_conditions(c, A, b)) < 1e-14
    c4, A4, b4 = wt.erk_tableau(wt.ERK_RK4)
    assert max(abs(r) for r in order_conditions(c4, A4, b4)[:8]) < 1e-15   # RK4: orders 1-4 only


@pytest.mark.parametrize("method,order", [(1, 5), (0, 4)])
@pytest.mark.parametrize("td", [False, True])
def test_time_convergence(O, method, order, td):
    o = O.OracleMesh(4, 2, A=0.05, outer_tag=7)
    x, y, z = o.coords()
    P0 = np.sin(2 * np.pi * x) * np.cos(np.pi * (y - z))
    Q0 = np.zeros(o.nn)
    bc = O.make_bc([2] * 6)
    if td:
        coef, tdb = None, (4, (0.2, 1.0), 0.0)
    else:
        coef, tdb = o.background(2, [0.05, 0.02, 0.1, 0.05, 0.5, 0.5, 0.5, 0.1, -0.1, 0.05, 0.2, 0.0, -0.15]), None
    T, dt = 0.24, 0.24 / 6
    run = lambda n: o.evolve_curved_erk(coef, P0, Q0, T / n, n, method=method, bc=bc, use_metric=True, td=tdb)[0]
    ref = run(96)
    e1, e2 = np.linalg.norm(run(6) - ref), np.linalg.norm(run(12) - ref)
    assert e1 / e2 > 2 ** order * 0.8, (e1, e2, e1 / e2)


def test_composed_tableau_keeps_the_order(wt):
    """Three RK4 steps of dt/3 written as one 12-stage explicit method: its Butcher
    tableau meets the order conditions up to 4 (the composition has RK4's order), it
    is strictly lower triangular, and its stage times are the substep times."""
    c, A, b = wt.erk_tableau(wt.ERK_RK4)
    C2, A2, B2 = wt.composed_tableau(c, A, b, 3)
    assert len(C2) == 12 <= wt.ERK_MAX_STAGES
    assert np.all(np.triu(A2) == 0)
    assert max(abs(r) for r in order_conditions(C2, A2, B2)[:8]) < 1e-15
    assert np.allclose(A2.sum(axis=1), C2, atol=1e-15)
