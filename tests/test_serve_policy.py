"""Host logic of the native request server (wt_serve_*), on the CPU: the
admission order of waiting requests (highest response ratio next, least work
first, arrival order; ties by arrival, then submission) against a restatement
of the three policies, the per-request device-byte estimate and precision
choice, and the victims of preemptive admission against a restatement of
that rule.  No device is touched."""
import random

import numpy as np

import pytest

from conftest import load_package


def restated_order(order, now, arrival, service, work):
    idx = list(range(len(arrival)))
    if order == 0:
        key = lambda k: (-(now - arrival[k] + service[k]) / service[k], arrival[k])
    elif order == 1:
        key = lambda k: (work[k], arrival[k])
    else:
        key = lambda k: arrival[k]
    return sorted(idx, key=key)  # stable: ties keep submission order


@pytest.mark.parametrize("order", [0, 1, 2])
def test_queue_order_matches_policy(order):
    wt = load_package()
    rng = random.Random(7 + order)
    for trial in range(200):
        n = rng.randint(0, 12)
        # coarse values so that ties in every key occur
        arrival = [rng.choice([0.0, 0.25, 0.5, 1.0]) for _ in range(n)]
        service = [rng.choice([0.1, 0.5, 2.0]) for _ in range(n)]
        work = [float(rng.choice([1, 4, 9])) for _ in range(n)]
        now = 1.5
        assert wt.serve_queue_order(order, now, arrival, service, work) == \
            restated_order(order, now, arrival, service, work), (trial, arrival, service, work)


def test_hrrn_favours_short_then_ages_long():
    wt = load_package()
    # both waiting since t = 0: the short request's ratio (wait + S) / S grows faster
    service, work = [20.0, 0.5], [1e12, 1e9]
    assert wt.serve_queue_order(wt.SERVE_HRRN, 1.0, [0.0, 0.0], service, work) == [1, 0]
    # a long request waiting since t = 0 against a short one waiting 0.1 s: the long
    # one's ratio (6 + 20) / 20 = 1.3 beats (0.1 + 0.5) / 0.5 = 1.2, so it is not starved
    assert wt.serve_queue_order(wt.SERVE_HRRN, 6.0, [0.0, 5.9], service, work) == [0, 1]
    assert wt.serve_queue_order(wt.SERVE_HRRN, 3.0, [0.0, 2.9], service, work) == [1, 0]
    arrival = [0.0, 2.9]
    assert wt.serve_queue_order(wt.SERVE_SJF, 10.0, arrival, service, work) == [1, 0]
    assert wt.serve_queue_order(wt.SERVE_FIFO, 10.0, arrival, service, work) == [0, 1]
    with pytest.raises(wt.WaveToyError):
        wt.serve_queue_order(3, 0.0, [0.0], [1.0], [1.0])
    with pytest.raises(wt.WaveToyError):
        wt.serve_queue_order(wt.SERVE_HRRN, 0.0, [0.0], [0.0], [1.0])


@pytest.mark.parametrize("prec,n,steps,bpn,want_prec", [
    (0, 8, 100, 520, 0), (0, 6, 100, 480, 0), (1, 8, 100, 340, 1), (1, 6, 900, 300, 1),
    (-1, 8, 250, 340, 1), (-1, 8, 251, 520, 0), (-1, 6, 2000, 480, 0)])
def test_cost_and_precision(prec, n, steps, bpn, want_prec):
    wt = load_package()
    d = wt.serve_desc(precision=prec, auto_fp32_max_steps=250)
    q = wt.serve_request(0.0, n, (3, 4, 5), warp_A=0.05, outer_tag=7, bg_kind=wt.BG_ADM_PERTURBED,
                         ic_params=wt.gaussian_params([(0.5, 0.5, 0.5)], [1.0], [0.1]), steps=steps,
                         bc3d=wt.make_bc3d([wt.BC_SOMMERFELD] * 6))
    nodes = 3 * 4 * 5 * n ** 3
    assert wt.serve_cost(d, q) == (float(nodes * (bpn + 272)), want_prec)


def test_request_validation():
    wt = load_package()
    d = wt.serve_desc()
    good = dict(arrival=0.0, N=6, M=2, steps=10)
    wt.serve_cost(d, wt.serve_request(**good))
    for bad in (dict(steps=0), dict(N=9), dict(M=0), dict(arrival=float("nan"))):
        with pytest.raises(wt.WaveToyError):
            wt.serve_cost(d, wt.serve_request(**{**good, **bad}))
    # time-dependent backgrounds are served (re-sampled every stage inside the batch)
    wt.serve_cost(d, wt.serve_request(**good, bg_kind=wt.BG_GAUGE_WAVE, bg_params=(0.1, 1.0, 0.0)))
    with pytest.raises(wt.WaveToyError):
        wt.serve_cost(wt.serve_desc(tick=0), wt.serve_request(**good))
    wt.serve_cost(wt.serve_desc(preempt=True), wt.serve_request(**good))
    bad_desc = wt.serve_desc(preempt=True)
    bad_desc.preempt = 2
    with pytest.raises(wt.WaveToyError):
        wt.serve_cost(bad_desc, wt.serve_request(**good))
    with pytest.raises(ValueError):
        wt.serve_request(**good, ic_params=[0.0] * 200)


def test_native_request_describes_build_solve():
    """serve.native_request carries the solve build_solve sets up: the warped cube
    (A = 0.05, Sommerfeld tag on every outer face), the seeded ADM background, the
    seeded Gaussian pulses of Phi, CFL 0.2 against the sampled speed bound."""
    wt = load_package()
    S, W = wt.serve, wt.workloads
    q = S.Request(rid=3, arrival=1.25, elements=5, n=6, steps=77, seed=41, scale=0.5, pulses=3)
    r = S.native_request(q)
    assert r.arrival == 1.25 and r.steps == 77 and r.cfl == 0.2
    assert (r.mesh.N, tuple(r.mesh.M), r.mesh.warp_A, r.mesh.outer_tag, r.mesh.periodic) == (6, (5, 5, 5), 0.05, 7, 0)
    p = W.adm_params(41, 0.5)
    assert r.bg.kind == wt.BG_ADM_PERTURBED and list(r.bg.p[:len(p)]) == [float(v) for v in p]
    c, a, w = W.pulses(41, 3, amp=(0.5, 1.0), width=(0.05, 0.15), centre=(0.25, 0.75))
    ic = wt.gaussian_params(c, a, w)
    assert r.ic_kind == wt.IC_GAUSSIANS and r.nic == len(ic) == 16 and list(r.ic[:r.nic]) == ic
    assert r.max_speed == W.max_speed(p, 24)
    assert list(r.bc.kinds) == [wt.BC_SOMMERFELD] * 6 and not r.bc.gPhi
    # the Python face of the engine charges what the engine's own estimate says
    srv = S.Server.__new__(S.Server)
    srv.budget, srv.tick, srv.max_active, srv.fill_nodes, srv.order = 1e12, 50, None, None, "hrrn"
    srv.precision, srv.fp32_form, srv.keep, srv.preempt = S.AUTO, wt.FP32_CUDA_CORES, False, False
    assert srv._cost(q) == q.nodes * (300 + 272)      # 77 steps <= the FP32 limit: FP32, n = 6


def preempt_choice_reference(budget, max_active, fill_nodes, used, nodes, left, cost, pre, hn, hl, hc):
    """Preemptive admission's victim rule, restated: running requests never preempted with at least
    twice the head's remaining work, most work first, as many as make room -- none if all do not."""
    def fits(u, na, run):
        return (u + hc <= budget and (max_active == 0 or na < max_active)
                and (fill_nodes == 0 or na == 0 or run < fill_nodes))
    work = [n * l for n, l in zip(nodes, left)]
    cand = sorted([k for k in range(len(nodes)) if pre[k] == 0 and work[k] >= 2.0 * hn * hl],
                  key=lambda k: -work[k])
    u, na, run, chosen = used, len(nodes), sum(nodes), []
    for k in cand:
        if fits(u, na, run):
            break
        u, na, run = u - cost[k], na - 1, run - nodes[k]
        chosen.append(k)
    return chosen if fits(u, na, run) else []


def test_preempt_choice_equals_the_rule():
    wt = load_package()
    rng = np.random.default_rng(11)
    picked = 0
    for _ in range(400):
        n = int(rng.integers(0, 7))
        nodes = [int(v) for v in rng.integers(1_000, 2_000_000, n)]
        left = [int(v) for v in rng.integers(1, 2000, n)]
        cost = [v * 600.0 for v in nodes]
        pre = [int(v) for v in rng.integers(0, 2, n)]
        budget = float(rng.uniform(1e9, 6e9))
        max_active = int(rng.integers(0, 5))
        fill = int(rng.choice([0, 1_000_000, 4_000_000]))
        used = float(sum(cost))
        hn, hl = int(rng.integers(1_000, 500_000)), int(rng.integers(1, 400))
        d = wt.serve_desc(hbm_budget=budget, max_active=max_active or None, fill_nodes=fill or None, preempt=True)
        got = wt.serve_preempt_choice(d, used, nodes, left, cost, pre, hn, hl, hn * 600.0)
        want = preempt_choice_reference(budget, max_active, fill, used, nodes, left, cost, pre, hn, hl, hn * 600.0)
        assert got == want
        picked += bool(got)
    assert picked > 20
