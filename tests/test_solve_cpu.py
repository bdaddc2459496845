"""CPU: the host side of wt_evolve3d (no device).

The sampling schedule follows the reference's loop (src/evolve.jl:1311-1318):
samples at range(t0, t1, Nt), fixed steps of dt while the integrator's time is
below the sample time, the time accumulated in T, and the integrator's stop at
t1 shortening a step that would pass it.  Here the library's schedule equals a
plain restatement of that loop on random spans, in Float64 and Float32; the
descriptor checks, node counts and the JSON-style configuration are checked too.
"""
import json

import numpy as np
import pytest


def reference_loop(t0, t1, nt, dt, T=float):
    """The sample loop, restated: steps before each sample, the last step, the times reached."""
    t0, t1, dt = T(t0), T(t1), T(dt)
    t, last, steps, ts = t0, dt, [], []
    for n in range(nt):
        target = t0 if n == 0 else t1 if n == nt - 1 else T(float(t0) + (float(t1) - float(t0)) * n / (nt - 1))
        k = 0
        while t < target:
            if T(t + dt) > t1:
                last, t = T(t1 - t), t1
            else:
                t = T(t + dt)
            k += 1
        steps.append(k)
        ts.append(float(t))
    return steps, float(last), ts


def test_schedule_small_case(wt):
    steps, last, ts = wt.solve_schedule(0.0, 1.0, 5, 0.3)
    assert list(steps) == [0, 1, 1, 1, 1]
    assert ts[-1] == 1.0 and ts[0] == 0.0
    assert last == pytest.approx(0.1, abs=1e-15) and last < 0.3
    # dt dividing the span: no step is shortened, every sample lands on its time
    steps, last, ts = wt.solve_schedule(0.0, 1.0, 3, 0.125)
    assert list(steps) == [0, 4, 4] and last == 0.125 and list(ts) == [0.0, 0.5, 1.0]
    # one sample: t0 only
    steps, last, ts = wt.solve_schedule(0.5, 2.0, 1, 0.1)
    assert list(steps) == [0] and list(ts) == [0.5]


@pytest.mark.parametrize("T,prec", [(float, 0), (np.float32, 1)])
def test_schedule_equals_the_reference_loop(wt, T, prec):
    rng = np.random.default_rng(3)
    for _ in range(200):
        t0 = float(rng.uniform(-1, 1))
        t1 = t0 + float(rng.uniform(0, 2))
        nt = int(rng.integers(1, 40))
        dt = float(rng.uniform(0.003, 0.4))
        s, last, ts = wt.solve_schedule(t0, t1, nt, dt, prec)
        rs, rlast, rts = reference_loop(t0, t1, nt, dt, T)
        assert list(s) == rs and list(ts) == rts and last == rlast, (t0, t1, nt, dt)


def test_schedule_rejects_bad_spans(wt):
    for args in ((1.0, 0.0, 3, 0.1), (0.0, 1.0, 0, 0.1), (0.0, 1.0, 3, 0.0), (0.0, 1.0, 3, float("nan")),
                 (0.0, 1e9, 3, 1e-6)):
        with pytest.raises(wt.WaveToyError):
            wt.solve_schedule(*args)


def test_solve_desc_checks_and_nodes(wt):
    d = wt.solve_desc(N=6, M=(2, 3, 4), background=wt.BG_ADM_PERTURBED, bg_params=wt.workloads.adm_params(1))
    assert wt.solve_desc_check(d) == ""
    import ctypes as C
    nn = C.c_longlong()
    assert wt.library().wt_solve_nodes(C.byref(d), C.byref(nn)) == 0 and nn.value == 6 ** 3 * 24
    p = wt.solve_desc(N=4, M=2, mesh_kind=wt.MESH_CUBED_CUBE, patch_params=(0.3,))
    assert wt.library().wt_solve_nodes(C.byref(p), C.byref(nn)) == 0 and nn.value == 7 * 8 * 64
    for kw, why in ((dict(Nt=0), "nt"), (dict(t0=1.0, t1=0.5), "t0"), (dict(cfl=0.0), "cfl"),
                    (dict(N=9), "N"), (dict(eps_KO=-1.0), "eps_ko"), (dict(T=5), "precision")):
        assert why in wt.solve_desc_check(wt.solve_desc(**kw)), kw
    with pytest.raises(ValueError):
        wt.solve_desc(bc3d=wt.make_bc3d([1] * 6, gPhi=object()))


def test_solve_config_from_json(wt, tmp_path):
    cfg = {"T": "Float32", "N": 8, "M": [4, 4, 2], "warp_A": 0.05, "background": "adm_perturbed",
           "bg_params": list(wt.workloads.adm_params(2)), "ic": "gaussians",
           "ic_params": wt.gaussian_params(*wt.workloads.pulses(2, 2)), "bc": {"kinds": [2] * 6},
           "eps_KO": 0.0, "t1": 0.25, "Nt": 11, "cfl": 0.2, "max_speed": 1.5}
    path = tmp_path / "solve.json"
    path.write_text(json.dumps(cfg))
    d = wt.load_solve_config(str(path))
    assert wt.solve_desc_check(d) == ""
    assert d.precision == wt.WT_F32 and d.mesh.N == 8 and list(d.mesh.M) == [4, 4, 2]
    assert d.bg.kind == wt.BG_ADM_PERTURBED and d.ic_kind == wt.IC_GAUSSIANS and d.nt == 11
    assert list(d.bc.kinds) == [2] * 6 and d.t1 == 0.25 and d.max_speed == 1.5
    with pytest.raises(ValueError):
        wt.solve_config({"mesh_kind": "torus"})


def test_bench_config_rejects_unknown_options(tmp_path):
    import os
    import subprocess
    import sys
    import conftest
    cfg = tmp_path / "bench.json"
    cfg.write_text(json.dumps({"workload": "serve", "rate": 0.6, "no_such_option": 1}))
    r = subprocess.run([sys.executable, os.path.join(conftest.ROOT, "bench.py"), "--config", str(cfg)],
                       capture_output=True, text=True, timeout=120)
    assert r.returncode == 2 and "no_such_option" in r.stderr


def build_slice_reference(x, y, z, yt, zt, atol):
    """_build_slice_3d (src/evolve.jl:104-123), restated: nodes strictly within atol of the line,
    in storage order, the first at each x kept, then sorted by x (stable)."""
    idx, xs = [], []
    for n in range(len(x)):
        if abs(y[n] - yt) < atol and abs(z[n] - zt) < atol:
            if not any(abs(x0 - x[n]) < atol for x0 in xs):
                idx.append(n)
                xs.append(x[n])
    perm = sorted(range(len(xs)), key=lambda q: xs[q])
    return [idx[q] for q in perm], [xs[q] for q in perm]


@pytest.mark.parametrize("N,M,A,atol", [(6, 4, 0.05, 1.4901161193847656e-08), (8, 2, 0.0, 1.4901161193847656e-08),
                                        (5, (4, 2, 2), 0.05, 3.4526698e-4)])
def test_slice_selection_equals_the_reference_rule(wt, O, N, M, A, atol):
    o = O.OracleMesh(N, M, A=A, outer_tag=7)
    x, y, z = o.coords()
    nodes, xs = wt.slice_select(np.stack([x, y, z], axis=1), 0.5, 0.5, atol)
    rn, rx = build_slice_reference(x, y, z, 0.5, 0.5, atol)
    assert list(nodes) == rn and list(xs) == rx
    assert len(rn) > 0 and np.all(np.diff(xs) > 0)
    raw = int(np.sum((np.abs(y - 0.5) < atol) & (np.abs(z - 0.5) < atol)))
    assert raw > len(rn)                       # shared face nodes appear once
