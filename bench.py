#!/usr/bin/env python
"""Benchmark: DOF-updates/s of the RK4-stepped 3D SBP-SAT ADM wave solve on B200.

Workload (default): warped cube (A = 0.05) with 64^3 elements and n = 8 GLL nodes
per axis (134,217,728 nodes), perturbed ADM background, eight seeded Gaussian
pulses, Sommerfeld outer faces, curvilinear split-form RHS, classic RK4 at CFL
0.2, FP64 (the plain drop-in form).  One step = one RK4 step over the whole
mesh; a DOF-update = one of (Phi, Pi) at one node advanced one step.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--elements M] [--n 8] [--precision f64|f32]

--impl reference times the CPU restatement of the path (the reference is Julia
and cannot run here) on the host cores, one bounded sample per step.  For N > 1
every rank runs its own independent solve (weak scaling, no collective on the
data path); timing is the max over ranks.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import math
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG_DIR = os.path.join(ROOT, "wavetoysecondorder.jl_b200")


def package():
    name = "wavetoy_b200"
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(name, os.path.join(PKG_DIR, "__init__.py"),
                                                  submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profiled_traffic(key: str):
    """DRAM bytes per node per launch of a kernel from the committed ncu summary
    (profiles/*.md lines 'traffic_bytes_per_node <key> = <value>'), or None."""
    d = os.path.join(ROOT, "profiles")
    if not os.path.isdir(d):
        return None
    for fn in sorted(os.listdir(d)):
        if not fn.endswith(".md"):
            continue
        for line in open(os.path.join(d, fn)):
            line = line.strip().strip("`")
            parts = line.replace("=", " = ").split()
            if len(parts) >= 4 and parts[0] == "traffic_bytes_per_node" and parts[1] == key and parts[2] == "=":
                try:
                    return float(parts[3])
                except ValueError:
                    pass
    return None


class ClockSampler:
    """nvidia-smi clocks/throttle sampling during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.samples = []
        self.proc = None
        self.thread = None

    def start(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 8:
                self.samples.append(parts)

    def stop(self):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if self.thread is not None:
            self.thread.join(timeout=2)
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = sorted(float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit())
        mx = max((float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()), default=None)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for s in self.samples for k in range(4) if s[4 + k].lower() == "active"})
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": mx, "reasons": reasons,
                "samples": len(self.samples)}


def FP32_FORMS(wt):
    """--fp32-form names of the FP32 precision forms."""
    return {"comp": wt.FP32_COMPENSATED, "bf16x3": wt.FP32_BF16X3, "bf16x2": wt.FP32_BF16X2,
            "cuda": wt.FP32_CUDA_CORES}


def cpu_model() -> str:
    """The host CPU's model name and logical core count (for the CPU baseline's record)."""
    name = "unknown"
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    name = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return f"{name}, {os.cpu_count()} logical cores"


def rank_seed(seed: int, rank: int) -> int:
    """Seed of rank `rank`'s independent solve (weak scaling: one solve per rank)."""
    return seed + 7919 * rank


def aggregate(dist, seconds: float, units: float, device: str = "cpu"):
    """Whole-job rate over all ranks: (sum of the units every rank processed) /
    (max over ranks of the device-timed seconds).  Returns (rate, max seconds,
    total units).  dist is torch.distributed (any backend) or None for one rank."""
    import torch
    t = torch.tensor([seconds], dtype=torch.float64, device=device)
    u = torch.tensor([units], dtype=torch.float64, device=device)
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.all_reduce(u, op=dist.ReduceOp.SUM)
    return float(u.item()) / float(t.item()), float(t.item()), float(u.item())


def workload_desc(args, nn):
    return {"workload": f"warped-cube ADM solve, {args.elements}^3 elements, n={args.n} "
                        f"({nn:,} nodes), Sommerfeld faces, curvilinear split form, RK4 CFL 0.2, "
                        f"{args.precision.upper()}",
            "elements_per_axis": args.elements, "n": args.n, "nodes": nn, "precision": args.precision,
            **({"fp32_form": args.fp32_form} if args.precision == "f32" else {}),
            "warp_A": 0.05, "eps_KO": 0.0, "seed": args.seed,
            "l2": "inputs larger than L2 (each field %.2f GB > 126 MB)" % (nn * (8 if args.precision == "f64" else 4) / 1e9)}


def cpu_sample(wt, O, args, seconds: float = 12.0, max_steps: int = 40):
    """Time the CPU oracle on a bounded sample of the workload: the 16^3-element
    cube of the same family (same n, background, pulses), RK4 steps until
    `seconds` elapse.  Returns (DOF-updates/s, cores, description)."""
    import numpy as np
    M = min(16, args.elements)
    m = O.OracleMesh(args.n, M, A=0.05, outer_tag=7)
    p = wt.workloads.adm_params(args.seed)
    coef = m.background(2, p)
    x, y, z = m.coords()
    c, a, w = wt.workloads.pulses(args.seed, 8, amp=(0.5, 1.0), width=(0.05, 0.15), centre=(0.25, 0.75))
    Phi = wt.workloads.gaussian_field(x, y, z, c, a, w)
    Pi = np.zeros_like(Phi)
    dt = 0.2 * m.min_spacing() / wt.workloads.max_speed(p)
    bc = O.make_bc([O.BC_SOMMERFELD] * 6)
    steps = 0
    t0 = time.perf_counter()
    while True:
        Phi, Pi = m.evolve_curved(coef, Phi, Pi, dt, 1, bc=bc, use_metric=True)
        steps += 1
        el = time.perf_counter() - t0
        if el >= seconds or steps >= max_steps:
            break
    return 2.0 * m.nn * steps / el, O.num_threads(), f"{M}^3 elements x {args.n}^3 nodes ({m.nn:,} nodes), " \
                                                     f"{steps} RK4 steps in {el:.1f} s"


def run_reference(args):
    """CPU arm: the oracle restatement (the Julia reference cannot run here)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    wt = package()
    sys.path.insert(0, ROOT)
    from oracle import oracle as O
    O.build()
    import numpy as np
    M = min(16, args.elements)
    m = O.OracleMesh(args.n, M, A=0.05, outer_tag=7)
    p = wt.workloads.adm_params(args.seed)
    coef = m.background(2, p)
    x, y, z = m.coords()
    c, a, w = wt.workloads.pulses(args.seed, 8, amp=(0.5, 1.0), width=(0.05, 0.15), centre=(0.25, 0.75))
    Phi = wt.workloads.gaussian_field(x, y, z, c, a, w)
    Pi = np.zeros_like(Phi)
    dt = 0.2 * m.min_spacing() / wt.workloads.max_speed(p)
    bc = O.make_bc([O.BC_SOMMERFELD] * 6)
    for _ in range(args.warmup):
        Phi, Pi = m.evolve_curved(coef, Phi, Pi, dt, 1, bc=bc, use_metric=True)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        Phi, Pi = m.evolve_curved(coef, Phi, Pi, dt, 1, bc=bc, use_metric=True)
    el = time.perf_counter() - t0
    value = 2.0 * m.nn * args.steps / el
    nn_full = args.n ** 3 * args.elements ** 3
    sample = f"each step: one RK4 step of the {M}^3-element x {args.n}^3-node sample ({m.nn:,} nodes) " \
             f"of the workload"
    line = {"impl": "reference", "metric": "DOF-updates/s", "value": value, "unit": "DOF-updates/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000.0 * el / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded ADM background, 8 Gaussian pulses)",
            "config": workload_desc(args, nn_full),
            "cpu_baseline": {"value": value, "unit": "DOF-updates/s", "cores": O.num_threads(), "kind": "port",
                             "cpu": cpu_model(), "sample_is_full_config": M == args.elements,
                             "sample": sample},
            "e2e": {"value": value, "unit": "DOF-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "the reference is Julia with unvendored dependencies (no toolchain here); its CPU path is "
                    "timed through the C++ Float64 restatement of the same arithmetic, all host threads"}
    print(json.dumps(line), flush=True)


def run_ours(args):
    import numpy as np
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    wt = package()
    ctx = wt.Context(local)
    prec = wt.WT_F64 if args.precision == "f64" else wt.WT_F32
    M, N = args.elements, args.n
    mesh = wt.Mesh.warped_uniform_hex(ctx, N, M, 0.0, 1.0, 0.05, outer_tag=wt.SOMMERFELD_BDRY_TAG, precision=prec)
    if prec == wt.WT_F32:
        mesh.set_fp32_form(FP32_FORMS(wt)[args.fp32_form])
    seed = rank_seed(args.seed, rank)
    p = wt.workloads.adm_params(seed)
    coef = wt.sample_background3d(mesh, wt.BG_ADM_PERTURBED, p)
    ws = wt.make_wave3d_workspace(mesh)
    if args.unfused:
        ws.set_fused(False)
    nn = mesh.nn
    Phi = mesh.zeros()
    Pi = mesh.zeros()
    c, a, w = wt.workloads.pulses(seed, 8, amp=(0.5, 1.0), width=(0.05, 0.15), centre=(0.25, 0.75))
    ic = wt.gaussian_params(c, a, w)
    wt.initial_state(ws, wt.IC_GAUSSIANS, ic, Phi, Pi)
    dt = 0.2 * mesh.min_spacing() / wt.workloads.max_speed(p)
    bc = wt.make_bc3d([wt.BC_SOMMERFELD] * 6)
    study = args.precision == "f64" and world == 1 and not args.no_precision_study
    E_0 = wt.wave3d_energy(Phi, Pi, coef, ws, metric=True) if study else None

    def step():
        wt.step_rk4_curved(Phi, Pi, coef, ws, dt, 1, eps_KO=0.0, bc3d=bc, metric=True)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    n0 = ctx.launch_count()
    ctx.profile(True)
    stream = torch.cuda.current_stream()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        step()
    ev1.record(stream)
    torch.cuda.synchronize()
    ctx.profile(False)
    (k1_ms, k1_n), (k2_ms, k2_n), (fk_ms, fk_n) = ctx.profile_read()
    launches = ctx.launch_count() - n0
    clocks = sampler.stop()
    t_ms = ev0.elapsed_time(ev1)
    if dist is not None:
        dist.barrier()
    value, t_max, _ = aggregate(dist, t_ms / 1000.0, 2.0 * nn * args.steps, "cuda")
    finite = not ctx.nonfinite()
    ref = None
    if study:
        # the reference of the FP32 forms: the FP64 state after the study's step count
        # (config C3: 200 steps), continued from the timed steps on a copy of the state
        Pr, Qr = Phi.clone(), Pi.clone()
        extra = max(0, args.study_steps - args.warmup - args.steps)
        if extra:
            wt.step_rk4_curved(Pr, Qr, coef, ws, dt, extra, eps_KO=0.0, bc3d=bc, metric=True)
        ref = (torch.cat([Pr, Qr]), wt.wave3d_energy(Pr, Qr, coef, ws, metric=True))
        del Pr, Qr
    alt = None
    if prec == wt.WT_F64 and N == 8:
        # the other stage form of the FP64 n = 8 step (fused stage kernel <-> two-kernel
        # stages), timed right after on copies of the state, so that both forms are
        # measured on the same GPU at nearly the same clocks
        P2, Q2 = Phi.clone(), Pi.clone()
        ws.set_fused(args.unfused)
        for _ in range(args.warmup):
            wt.step_rk4_curved(P2, Q2, coef, ws, dt, 1, eps_KO=0.0, bc3d=bc, metric=True)
        torch.cuda.synchronize()
        asampler = ClockSampler(local)
        asampler.start()
        time.sleep(0.3)
        ctx.profile(True)
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a0.record(stream)
        for _ in range(args.steps):
            wt.step_rk4_curved(P2, Q2, coef, ws, dt, 1, eps_KO=0.0, bc3d=bc, metric=True)
        a1.record(stream)
        torch.cuda.synchronize()
        ctx.profile(False)
        aclocks = asampler.stop()
        pa = ctx.profile_read()
        ta = a0.elapsed_time(a1) / 1000.0
        alt = {"form": "fused stage kernel (wt_workspace_set_fused)" if args.unfused else "two-kernel stages",
               "value": 2.0 * nn * args.steps / ta, "unit": "DOF-updates/s", "ms_per_step": 1000.0 * ta / args.steps,
               "ratio_to_value": (2.0 * nn * args.steps / ta) / (2.0 * nn * args.steps / (t_ms / 1000.0)),
               "kernels_ms_per_launch": {k: (m / n if n else None) for k, (m, n) in
                                         zip(("k_cons_k1", "k_cons_k2", "k_cons_fk_n8"), pa)},
               "clocks": aclocks}
        ws.set_fused(not args.unfused)
        del P2, Q2
    ko = None
    if prec == wt.WT_F64 and N == 8 and world == 1:
        # Kreiss-Oliger dissipation on (eps_KO = 0.1, the reference's wave3d_curved_rhs!
        # with the line-local D^6 passes): RK4 steps of the same solve on copies of the
        # state; mu (the power iteration) is computed before the timed steps
        P2, Q2 = Phi.clone(), Pi.clone()
        _ = ws.mu
        for _ in range(2):
            wt.step_rk4_curved(P2, Q2, coef, ws, dt, 1, eps_KO=0.1, bc3d=bc, metric=True)
        torch.cuda.synchronize()
        kst = max(3, args.steps // 4)
        k0, k1e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        k0.record(stream)
        for _ in range(kst):
            wt.step_rk4_curved(P2, Q2, coef, ws, dt, 1, eps_KO=0.1, bc3d=bc, metric=True)
        k1e.record(stream)
        torch.cuda.synchronize()
        tk = k0.elapsed_time(k1e) / 1000.0
        ko = {"eps_KO": 0.1, "steps": kst, "value": 2.0 * nn * kst / tk, "unit": "DOF-updates/s",
              "ms_per_step": 1000.0 * tk / kst, "ratio_to_value": (2.0 * nn * kst / tk) / value,
              "finite": bool(torch.isfinite(P2).all() and torch.isfinite(Q2).all())}
        del P2, Q2

    # end to end through the host-buffer API (wt_evolve_curved_host, the shape of
    # evolve3d): page-locked host state in, one RK4 step per sample, state and
    # energy back to the host after every step (the library overlaps each
    # sample's device-to-host copy with the next sample's step)
    hdt = torch.float64 if prec == wt.WT_F64 else torch.float32
    wb = 8 if prec == wt.WT_F64 else 4
    Ph = torch.empty(nn, dtype=hdt, pin_memory=True)
    Qh = torch.empty(nn, dtype=hdt, pin_memory=True)
    Ph.copy_(Phi.cpu())
    Qh.copy_(Pi.cpu())
    E = np.zeros(args.steps)
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    t0 = time.perf_counter()
    wt.evolve_curved_host(Ph, Qh, coef, ws, dt, 1, args.steps, bc3d=bc, metric=True, energy=E)
    te = torch.tensor([time.perf_counter() - t0], dtype=torch.float64, device="cuda")
    if dist is not None:
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
    te = float(te.item())
    e2e = {"value": 2.0 * nn * args.steps * world / te, "unit": "DOF-updates/s",
           "h2d_bytes_per_step": int(2 * nn * wb / args.steps), "d2h_bytes_per_step": int(2 * nn * wb + 8),
           "api": ("wt_evolve_curved_host" if prec == wt.WT_F64 else "wt_evolve_curved_host_f32")
           + " (evolve3d shape: state and energy copied to page-locked host buffers every step)"}
    # the host link that bounds it: one device-to-host copy of both state fields into the
    # page-locked buffers, timed with CUDA events on the current stream
    hs = torch.cuda.current_stream()
    l0, l1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    Ph.copy_(Phi, non_blocking=True)   # warm
    torch.cuda.synchronize()
    l0.record(hs)
    Ph.copy_(Phi, non_blocking=True)
    Qh.copy_(Pi, non_blocking=True)
    l1.record(hs)
    torch.cuda.synchronize()
    link = 2 * nn * wb / (l0.elapsed_time(l1) / 1000.0) / 1e9
    step_s = te / args.steps   # seconds per step end to end
    e2e["d2h_link_GBps"] = link
    e2e["d2h_bound_frac"] = (e2e["d2h_bytes_per_step"] / step_s / 1e9) / link
    del Ph, Qh

    # roofline of the dominant kernel: the fused stage kernel (FP64 n = 8: three of
    # its launches per step), else K1 (gradient + flux + Phi stage update)
    hbm, src = peaks()
    wbytes = 8 if prec == wt.WT_F64 else 4
    fused = fk_n > 0
    # K1 in the two-kernel step: Phi, Pi, 20 coefficient words, F (3), Phi RK stage
    # words (3, the mean over the four stages); the fused step's K1_0 (stage 0)
    # reads no RK state: Phi, Pi, 20 coefficient words, F (3), stage value, acc
    k1_words = 1 + 1 + 20 + 3 + (2 if fused else 3)
    k1_avg_s = (k1_ms / max(k1_n, 1)) / 1000.0
    k1_achieved = k1_words * wbytes * nn / k1_avg_s / 1e9 if k1_n else None
    # fused stage FK_s, s = 0, 1, 2 (mean): K2 half F_s (3), Ja (9), 1/J, Pi state y and acc
    # read (5/3), acc written (1); K1 half Phi_{s+1} (1), ten coefficients, Phi y and acc read
    # (5/3), F_{s+1} (3) and the Phi stage value or state (1) written, acc written (2/3)
    fk_words = 3 + 9 + 1 + 5 / 3 + 1 + 1 + 10 + 5 / 3 + 3 + 1 + 2 / 3
    fk_avg_s = (fk_ms / max(fk_n, 1)) / 1000.0
    fk_achieved = fk_words * wbytes * nn / fk_avg_s / 1e9 if fk_n else None
    k2_avg_s = (k2_ms / max(k2_n, 1)) / 1000.0
    # K2: F (3), Ja (9), 1/J, Pi RK stage words (3, four-stage mean; the fused step's
    # K2_3 reads acc and writes the state: 2)
    k2_words = 3 + 10 + (2 if fused else 3)
    if fused:
        traffic_pn = profiled_traffic("fk_curv_f64")
        rl_kernel, rl_words, rl_achieved, rl_avg_s = (
            "k_cons_fk_n8 (fused stage: divergence + Pi stage s, gradient + flux + Phi stage s + 1)", fk_words,
            fk_achieved, fk_avg_s)
    else:
        traffic_pn = profiled_traffic(f"k1_curv_{args.precision}" if args.precision == "f64" or args.fp32_form == "cuda"
                                      else f"k1_curv_f32_{args.fp32_form}")
        rl_kernel, rl_words, rl_achieved, rl_avg_s = (
            "k_cons_k1 (split-form gradient + flux + Phi RK4 stage)", k1_words, k1_achieved, k1_avg_s)
    step_bytes = wbytes * (34 + 4 * 20) * nn
    line = {
        "metric": "DOF-updates/s", "value": value, "unit": "DOF-updates/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1000.0 * t_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": args.precision,
        "data": "synthetic (seeded ADM background, 8 seeded Gaussian pulses; no dataset)",
        "config": workload_desc(args, nn),
        "roofline": {"bound": "hbm", "kernel": rl_kernel,
                     "achieved": rl_achieved, "peak": hbm, "unit": "GB/s",
                     "frac": (rl_achieved / hbm) if rl_achieved else None,
                     "traffic": (traffic_pn * nn) if traffic_pn else None,
                     "algorithmic_bytes_per_launch": rl_words * wbytes * nn,
                     "avg_launch_ms": 1000.0 * rl_avg_s, "peak_source": f"{src} (MEASURED_PEAKS.json hbm_gbs)"},
        "kernels": {"k_cons_k1": {"launches": k1_n, "ms": k1_ms,
                                  "achieved_GBps": k1_achieved},
                    "k_cons_k2": {"launches": k2_n, "ms": k2_ms,
                                  "achieved_GBps": k2_words * wbytes * nn / k2_avg_s / 1e9 if k2_n else None},
                    "k_cons_fk_n8": {"launches": fk_n, "ms": fk_ms, "achieved_GBps": fk_achieved}},
        "step_roofline": {"algorithmic_bytes_per_step": step_bytes,
                          "achieved_GBps": step_bytes / (t_max / args.steps) / 1e9,
                          "frac": step_bytes / (t_max / args.steps) / 1e9 / hbm,
                          "definition": "w (34 + 4 C) bytes per node per RK4 step, C = 20 streamed coefficient words"},
        "e2e": e2e, "gpu_launches": launches, "clocks": clocks, "finite": finite,
    }
    if alt is not None:
        line["other_stage_form"] = alt
    if ko is not None:
        line["ko_step"] = ko
    if study:
        # the precision study of the large solve: every FP32 form on the same workload,
        # timed like the FP64 form and compared with its state after the same steps
        ws.close(); coef.close(); mesh.close()
        del Phi, Pi
        torch.cuda.empty_cache()
        line["precision_forms"] = precision_study(wt, ctx, args, seed, p, ic, dt, ref, E_0, value, hbm)
        comp = line["precision_forms"]["fp32_compensated"]
        line["chosen_form"] = {
            "form": "fp32_compensated (the chosen split-precision form: FP32 storage, compensated Phi, "
                    "FP64 gradient of Phi)",
            "dof_updates_per_s": comp["value"], "speedup_vs_plain_f64": comp["speedup_vs_f64"],
            "rel_l2_vs_f64": comp["rel_l2_vs_f64"], "step_roofline_frac": comp["step_roofline"]["frac"],
            "target": "speedup >= 3 at step_roofline_frac >= 0.7, rel_l2_vs_f64 <= 1e-5"}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        sys.path.insert(0, ROOT)
        from oracle import oracle as O
        O.build()
        v, cores, sample = cpu_sample(wt, O, args)
        line["cpu_baseline"] = {"value": v, "unit": "DOF-updates/s", "cores": cores, "kind": "port",
                                "cpu": cpu_model(), "sample_is_full_config": args.elements <= 16,
                                "sample": sample}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def precision_study(wt, ctx, args, seed, p, ic, dt64, ref, E64_0, value64, hbm):
    """The FP32 forms on the large solve (same mesh, background, initial data and
    steps as the FP64 form): per form DOF-updates/s over the timed steps, the step
    roofline against w (34 + 4 C) bytes with w = 4, the speed-up over the FP64
    form, and the relative L2 / max error against the FP64 state and the energy
    drift after --study-steps steps (the timed ones included)."""
    import torch
    M, N = args.elements, args.n
    mesh = wt.Mesh.warped_uniform_hex(ctx, N, M, 0.0, 1.0, 0.05, outer_tag=wt.SOMMERFELD_BDRY_TAG, precision=wt.WT_F32)
    coef = wt.sample_background3d(mesh, wt.BG_ADM_PERTURBED, p)
    ws = wt.make_wave3d_workspace(mesh)
    nn = mesh.nn
    dt = 0.2 * mesh.min_spacing() / wt.workloads.max_speed(p)
    assert dt == dt64
    bc = wt.make_bc3d([wt.BC_SOMMERFELD] * 6)
    Phi, Pi = mesh.zeros(), mesh.zeros()
    refv, E64 = ref
    out = {}
    for name, form in (("fp32_compensated", wt.FP32_COMPENSATED), ("fp32_cuda_cores", wt.FP32_CUDA_CORES),
                       ("fp32_bf16x3", wt.FP32_BF16X3)):
        mesh.set_fp32_form(form)
        wt.initial_state(ws, wt.IC_GAUSSIANS, ic, Phi, Pi)
        E0 = wt.wave3d_energy(Phi, Pi, coef, ws, metric=True)
        for _ in range(args.warmup):
            wt.step_rk4_curved(Phi, Pi, coef, ws, dt, 1, bc3d=bc, metric=True)
        torch.cuda.synchronize()
        ctx.profile(True)
        stream = torch.cuda.current_stream()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            wt.step_rk4_curved(Phi, Pi, coef, ws, dt, 1, bc3d=bc, metric=True)
        e1.record(stream)
        torch.cuda.synchronize()
        ctx.profile(False)
        (k1_ms, k1_n), (k2_ms, k2_n), _ = ctx.profile_read()
        t_s = e0.elapsed_time(e1) / 1000.0
        v = 2.0 * nn * args.steps / t_s
        extra = max(0, args.study_steps - args.warmup - args.steps)   # untimed, up to the study's step count
        if extra:
            wt.step_rk4_curved(Phi, Pi, coef, ws, dt, extra, bc3d=bc, metric=True)
        step_bytes = 4 * (34 + 4 * 20) * nn
        x = torch.cat([Phi, Pi]).double()
        d = x - refv
        E = wt.wave3d_energy(Phi, Pi, coef, ws, metric=True)
        out[name] = {
            "value": v, "unit": "DOF-updates/s", "ms_per_step": 1000.0 * t_s / args.steps,
            "speedup_vs_f64": v / value64,
            "step_roofline": {"algorithmic_bytes_per_step": step_bytes,
                              "frac": step_bytes / (t_s / args.steps) / 1e9 / hbm},
            "kernels_ms_per_launch": {"k1": k1_ms / max(k1_n, 1), "k2": k2_ms / max(k2_n, 1)},
            "rel_l2_vs_f64": float(torch.linalg.norm(d) / torch.linalg.norm(refv)),
            "max_err_vs_f64": float(d.abs().max() / refv.abs().max()),
            "energy_drift": E / E0 - 1.0, "steps_compared": max(args.study_steps, args.warmup + args.steps),
            "finite": not ctx.nonfinite()}
    out["f64_energy_drift"] = E64 / E64_0 - 1.0
    ws.close(); coef.close(); mesh.close()
    torch.cuda.empty_cache()
    return out


def run_slab(args):
    """One solve split across ranks: the --elements^3 warped ADM solve of the default
    workload with its z element layers partitioned into one slab per rank
    (slabs.py: a ghost layer beyond each cut, one halo exchange per RK4 stage of
    the face planes the owned elements read across each cut -- or, with
    --layer-halo, of whole layers -- NCCL point-to-point between GPUs; device
    copies between slabs on one GPU).  Strong scaling: the whole solve's DOF-updates over the maximum of
    the ranks' device times."""
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    wt = package()
    S = wt.slabs
    ctx = wt.Context(local)
    prec = wt.WT_F64 if args.precision == "f64" else wt.WT_F32
    M, N = args.elements, args.n
    form = FP32_FORMS(wt)[args.fp32_form]
    # one slab per rank; on one GPU, --slabs slabs in this process (exchanged by device copies)
    nslabs = world if world > 1 else max(1, args.slabs)
    parts = S.partition(M, nslabs)
    mine = [parts[rank]] if world > 1 else parts
    p = wt.workloads.adm_params(args.seed)
    c, a, w = wt.workloads.pulses(args.seed, 8, amp=(0.5, 1.0), width=(0.05, 0.15), centre=(0.25, 0.75))
    slabs = []
    for r in mine:
        sl = S.Slab(ctx, r, N, M, warp_A=0.05, outer_tag=wt.SOMMERFELD_BDRY_TAG, precision=prec,
                    bg_kind=wt.BG_ADM_PERTURBED, bg_params=p, fp32_form=form if prec == wt.WT_F32 else None)
        wt.initial_data(sl.mesh, wt.IC_GAUSSIANS, wt.gaussian_params(c, a, w), sl.Phi)
        slabs.append(sl)
    h = torch.tensor([min(sl.mesh.min_spacing() for sl in slabs)], dtype=torch.float64, device="cuda")
    if dist is not None:
        dist.all_reduce(h, op=dist.ReduceOp.MIN)
    dt = 0.2 * float(h.item()) / wt.workloads.max_speed(p)
    bc = wt.make_bc3d([wt.BC_SOMMERFELD] * 6)
    if args.layer_halo:   # every slab layer computed, whole layers exchanged after the first half
        halo = S.DistHalo(slabs[0], dist) if dist is not None else S.LocalHalo(slabs)
        stepper = S.step
    else:                 # owned layers only, face planes exchanged under the interior's first half
        halo = S.DistFaceHalo(slabs[0], dist) if dist is not None else S.LocalFaceHalo(slabs)
        stepper = S.step_faces
    stepper(slabs, halo, dt, args.warmup, bc)
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    n0 = ctx.launch_count()
    stream = torch.cuda.current_stream()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    stepper(slabs, halo, dt, args.steps, bc)
    ev1.record(stream)
    torch.cuda.synchronize()
    launches = ctx.launch_count() - n0
    clocks = sampler.stop()
    t_ms = ev0.elapsed_time(ev1)
    if dist is not None:
        dist.barrier()
    nodes = M ** 3 * N ** 3
    _, t_max, _ = aggregate(dist, t_ms / 1000.0, 0.0, "cuda")
    finite = not ctx.nonfinite()
    wb = 8 if prec == wt.WT_F64 else 4
    rng = mine[0]
    halo_bytes = ((wt.halo_size(slabs[0].ws) if args.layer_halo else wt.halo_face_size(slabs[0].ws)) * wb
                  if nslabs > 1 else 0)
    line = {
        "metric": "DOF-updates/s", "value": 2.0 * nodes * args.steps / t_max, "unit": "DOF-updates/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * t_max / args.steps,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": args.precision,
        "data": "synthetic (seeded ADM background, 8 seeded Gaussian pulses; no dataset)",
        "config": {**workload_desc(args, nodes),
                   "parallelism": f"z-slabs x{nslabs}" + (" (one per rank)" if world > 1 else " in one process"),
                   "halo": ("whole ghost layers, every slab layer computed" if args.layer_halo else
                            "shared face planes, owned layers only, exchange under the interior layers' first half"),
                   "layers_per_slab": [r.nown for r in parts],
                   "ghost_layers_rank0": rng.ghost_lo + rng.ghost_hi,
                   "halo_bytes_per_message": halo_bytes,
                   "messages_per_stage_per_rank": (rng.ghost_lo + rng.ghost_hi) * 2},
        "gpu_launches": launches, "clocks": clocks, "finite": finite,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    for sl in slabs:
        sl.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def run_batch(args):
    """Batched uneven solves: args.solves warped-cube solves (e ~ U{4..24}, n ~ {4,6,8},
    flat or perturbed ADM), the compensated FP32 form, advanced together by the
    batch (work-list kernels, CUDA graph per RK4 step, autotuned CTA shapes) for
    args.batch_steps steps; beside it the per-solve loops of the plain FP64, the
    plain FP32 and the compensated FP32 forms over the same solves."""
    import numpy as np
    import torch
    wt = package()
    S = wt.serve
    ctx = wt.Context(0)
    specs = wt.workloads.batch_specs(args.seed, args.solves)
    reqs = [S.Request(rid=k, arrival=0.0, elements=d["elements"], n=d["n"], steps=args.batch_steps, seed=d["seed"],
                      scale=d["scale"], pulses=2) for k, d in enumerate(specs)]
    t_setup = time.perf_counter()
    solves = [S.build_solve(ctx, q, wt.WT_F32) for q in reqs]
    t_setup = time.perf_counter() - t_setup
    batch = wt.Batch(ctx)
    bc = wt.make_bc3d([wt.BC_SOMMERFELD] * 6)
    for (mesh, coef, ws, Phi, Pi, dt) in solves:
        batch.add(Phi, Pi, coef, ws, dt, bc)
    nodes = sum(m.nn for (m, *_r) in solves)
    batch.step(args.warmup)  # builds the work lists, tunes, captures the graph
    torch.cuda.synchronize()
    sampler = ClockSampler(0)
    sampler.start()
    time.sleep(0.3)
    n0 = ctx.launch_count()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    batch.step(args.batch_steps)
    ev1.record()
    torch.cuda.synchronize()
    clocks = sampler.stop()
    t = ev0.elapsed_time(ev1) / 1000.0
    launches = ctx.launch_count() - n0
    groups = batch.groups()
    finite = not ctx.nonfinite()
    value = 2.0 * nodes * args.batch_steps / t
    # per-solve loops of the plain forms over every solve of the batch, 20 steps each
    order = sorted(range(len(reqs)), key=lambda k: reqs[k].nodes)
    batch.close()
    for objs in solves:
        for o in (objs[2], objs[1], objs[0]):
            o.close()
    del solves
    torch.cuda.empty_cache()
    loops = {}
    err = 0.0
    for prec, form, name in ((wt.WT_F64, None, "plain_fp64_per_solve_loop"),
                             (wt.WT_F32, wt.FP32_CUDA_CORES, "plain_fp32_per_solve_loop"),
                             (wt.WT_F32, wt.FP32_COMPENSATED, "compensated_fp32_per_solve_loop")):
        dof, secs = 0.0, 0.0
        for q in reqs:
            mesh, coef, ws, Phi, Pi, dt = S.build_solve(ctx, q, prec, form if form is not None else wt.FP32_COMPENSATED,
                                                        release=False)
            nst = 20
            wt.step_rk4_curved(Phi, Pi, coef, ws, dt, 3, bc3d=bc, metric=True)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for _ in range(nst):
                wt.step_rk4_curved(Phi, Pi, coef, ws, dt, 1, bc3d=bc, metric=True)
            torch.cuda.synchronize()
            secs += time.perf_counter() - t0
            dof += 2.0 * mesh.nn * nst
            for o in (ws, coef, mesh):
                o.close()
        loops[name] = {"value": dof / secs, "unit": "DOF-updates/s",
                       "sample": f"all {len(reqs)} solves, 20 steps each, one step_rk4_curved call per step"}
    # the small solves alone (e <= 8), where one launch per solve leaves the GPU mostly idle:
    # batched against the per-solve loop of the same (compensated) form
    small = [q for q in reqs if q.elements <= 8]
    sub = [S.build_solve(ctx, q, wt.WT_F32) for q in small]
    bs = wt.Batch(ctx)
    for (mesh, coef, ws, Phi, Pi, dt) in sub:
        bs.add(Phi, Pi, coef, ws, dt, bc)
    bs.step(3)
    torch.cuda.synchronize()
    e0s, e1s = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0s.record()
    bs.step(20)
    e1s.record()
    torch.cuda.synchronize()
    small_nodes = sum(m.nn for (m, *_r) in sub)
    v_small = 2.0 * small_nodes * 20 / (e0s.elapsed_time(e1s) / 1000.0)
    bs.close()
    dof, secs = 0.0, 0.0
    for (mesh, coef, ws, Phi, Pi, dt) in sub:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(20):
            wt.step_rk4_curved(Phi, Pi, coef, ws, dt, 1, bc3d=bc, metric=True)
        torch.cuda.synchronize()
        secs += time.perf_counter() - t0
        dof += 2.0 * mesh.nn * 20
    for objs in sub:
        for o in (objs[2], objs[1], objs[0]):
            o.close()
    del sub
    torch.cuda.empty_cache()
    small_line = {"solves": len(small), "nodes": small_nodes, "batched": v_small, "per_solve_loop": dof / secs,
                  "speedup": v_small / (dof / secs), "unit": "DOF-updates/s",
                  "note": "the solves with e <= 8 elements per axis, 20 steps, compensated FP32 form"}
    # split-precision accuracy on two small solves: batched FP32 vs the FP64 form after all steps
    for k in order[:2]:
        q = reqs[k]
        runs = []
        for prec in (wt.WT_F32, wt.WT_F64):
            mesh, coef, ws, Phi, Pi, dt = S.build_solve(ctx, q, prec, release=False)
            b = wt.Batch(ctx)
            b.add(Phi, Pi, coef, ws, dt, bc)
            b.step(args.batch_steps)
            runs.append(torch.cat([Phi, Pi]).double().cpu().numpy())
            b.close()
        err = max(err, float(np.linalg.norm(runs[0] - runs[1]) / np.linalg.norm(runs[1])))
    line = {"metric": "DOF-updates/s", "value": value, "unit": "DOF-updates/s", "n_gpus": 1,
            "steps": args.batch_steps, "warmup": args.warmup,
            "ms_per_step": 1000.0 * t / args.batch_steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 (compensated form: FP32 storage, compensated Phi, FP64 gradient of Phi)",
            "data": "synthetic (seeded solves; no dataset)",
            "config": {"workload": f"{len(reqs)} batched warped-cube solves, e~U{{4..24}}, n~{{4,6,8}}, flat or "
                                   f"ADM U(0,0.15), {nodes:,} nodes in total",
                       "solves": len(reqs), "nodes": nodes, "setup_s": t_setup,
                       "groups": [{"n": g[0], "n8_path": g[2], "epb_variant": g[3], "tiles": g[4]} for g in groups]},
            "gpu_launches": launches, "clocks": clocks, "finite": finite,
            "rel_l2_vs_fp64_after_all_steps": err, **loops,
            "speedup_vs_compensated_fp32_per_solve_loop": value / loops["compensated_fp32_per_solve_loop"]["value"],
            "speedup_vs_plain_fp64_per_solve_loop": value / loops["plain_fp64_per_solve_loop"]["value"],
            "small_solves": small_line}
    print(json.dumps(line), flush=True)


def run_serve(args):
    """Served solves: args.requests Poisson arrivals (e log-uniform in [4,32],
    n ~ {6,8}, 200..2000 steps) served by the continuous-batching server under
    a 150 GB budget in three forms: the compensated FP32 form for every request
    (the chosen form), FP64 for every request (the same continuous batching), and
    the plain FP64 per-request form (one solve at a time, in arrival order, as one
    evolve3d call per request).  Every served result is compared with the plain
    FP64 result of the same request."""
    import torch
    wt = package()
    S = wt.serve
    ctx = wt.Context(0)
    reqs = [S.Request.from_dict(d) for d in wt.workloads.serve_requests(args.seed, args.requests, args.rate)]
    out = {}
    # the served forms admit by response ratio (Server's default); the plain form runs
    # one request at a time in arrival order
    forms = (("plain_fp64_per_request", wt.WT_F64, 1, "fifo", False),
             ("served_fp32_compensated", wt.WT_F32, None, "hrrn", False),
             ("served_fp64", wt.WT_F64, None, "hrrn", False))
    if args.serve_chosen_only:   # a longer stream: the chosen form alone, FP64 checks on a sample
        forms = forms[1:2]
    if args.preempt:   # the chosen form without and with preemptive admission, compared bit for bit
        forms = forms[1:2] + (("served_fp32_compensated_preemptive", wt.WT_F32, None, "hrrn", True),)
    ref = {}
    first = {}
    for name, prec, max_active, order, preempt in forms:
        server = S.Server(ctx, precision=prec, hbm_budget=150e9, tick=50, max_active=max_active, keep_results=True,
                          order=order, fp32_form=wt.FP32_COMPENSATED, preempt=preempt)
        t0 = time.perf_counter()
        res = server.run(reqs)
        makespan = time.perf_counter() - t0
        out[name] = S.summary(res, makespan)
        if name == "plain_fp64_per_request":
            ref = {r.rid: torch.cat([r.Phi, r.Pi]).double() for r in res}
        elif args.preempt:
            # preemption changes when a request runs, not what it computes
            if not preempt:
                first = {r.rid: torch.cat([r.Phi, r.Pi]) for r in res}
            else:
                out[name]["bitwise_equal_to_non_preemptive"] = int(
                    sum(bool(torch.equal(torch.cat([r.Phi, r.Pi]), first[r.rid])) for r in res))
                out[name]["preempted_requests"] = int(sum(r.preemptions > 0 for r in res))
        elif args.serve_chosen_only:
            # every k-th request solved again alone in FP64 (the same set-up and steps)
            k = max(1, len(res) // 50)
            byrid = {q.rid: q for q in reqs}
            errs = []
            for r in sorted(res, key=lambda r: r.rid)[::k]:
                q = byrid[r.rid]
                mesh, coef, ws, P64, Q64, dt = S.build_solve(ctx, q, wt.WT_F64)
                wt.step_rk4_curved(P64, Q64, coef, ws, dt, q.steps, bc3d=wt.make_bc3d([wt.BC_SOMMERFELD] * 6),
                                   metric=True)
                x64 = torch.cat([P64, Q64])
                x = torch.cat([r.Phi, r.Pi]).double()
                errs.append(float(torch.linalg.norm(x - x64) / torch.linalg.norm(x64)))
                ws.close(); coef.close(); mesh.close()
            out[name]["fp64_checked_sample"] = len(errs)
            out[name]["max_rel_l2_vs_fp64"] = max(errs)
            out[name]["median_rel_l2_vs_fp64"] = sorted(errs)[len(errs) // 2]
            out[name]["sample_within_1e-5"] = int(sum(e <= 1e-5 for e in errs))
        else:
            errs = []
            for r in res:
                x = torch.cat([r.Phi, r.Pi]).double()
                errs.append(float(torch.linalg.norm(x - ref[r.rid]) / torch.linalg.norm(ref[r.rid])))
            out[name]["max_rel_l2_vs_fp64"] = max(errs)
            out[name]["median_rel_l2_vs_fp64"] = sorted(errs)[len(errs) // 2]
            out[name]["requests_within_1e-5"] = int(sum(e <= 1e-5 for e in errs))
            byrid = {q.rid: q for q in reqs}
            out[name]["over_1e-5"] = [
                {"rid": r.rid, "elements": byrid[r.rid].elements, "n": byrid[r.rid].n, "steps": byrid[r.rid].steps,
                 "final_time": round(r.dt * byrid[r.rid].steps, 3), "rel_l2": e}
                for r, e in zip(res, errs) if e > 1e-5]
        del res
        torch.cuda.empty_cache()
    main_ = out["served_fp32_compensated"]
    plain = out.get("plain_fp64_per_request")
    line = {"metric": "served solves/s", "value": main_["solves_per_s"], "unit": "solves/s", "n_gpus": 1,
            "steps": None, "warmup": 0, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 (compensated form: FP32 storage, compensated Phi, FP64 gradient of Phi)",
            "data": "synthetic (seeded Poisson request stream; no dataset)",
            "config": {"workload": f"{len(reqs)} served warped-cube solves, Poisson rate {args.rate}/s, "
                                   "e log-U[4,32], n~{6,8}, 200..2000 steps, 150 GB budget",
                       "requests": len(reqs), "rate_per_s": args.rate},
            "p50_latency_s": main_["p50_latency_s"], "p99_latency_s": main_["p99_latency_s"],
            "dof_updates_per_s": main_["dof_updates_per_s"],
            "speedup_vs_plain_fp64_solves_per_s": main_["solves_per_s"] / plain["solves_per_s"] if plain else None,
            **out, "finite": not ctx.nonfinite()}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--elements", type=int, default=64, help="elements per axis")
    ap.add_argument("--n", type=int, default=8, help="GLL nodes per axis")
    ap.add_argument("--precision", choices=["f64", "f32"], default="f64")
    ap.add_argument("--fp32-form", choices=["comp", "bf16x3", "bf16x2", "cuda"], default="comp",
                    help="FP32 form: compensated (default; FP64 gradient of the compensated Phi), plain CUDA cores, or split BF16 tensor cores "
                         "(three / two terms)")
    ap.add_argument("--seed", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--unfused", action="store_true",
                    help="FP64 n = 8: step through the two-kernel stages instead of the fused stage kernel")
    ap.add_argument("--study-steps", type=int, default=200,
                    help="precision study: RK4 steps after which each FP32 form is compared with FP64 (config C3: 200)")
    ap.add_argument("--no-precision-study", action="store_true",
                    help="skip the FP32 forms run after the FP64 line (default workload, one GPU)")
    ap.add_argument("--workload", choices=["solve", "batch", "serve", "slab"], default="solve",
                    help="solve: the large warped ADM solve (default; one independent solve per rank); "
                         "batch: batched uneven solves; serve: served Poisson request stream; slab: the "
                         "large solve split into one z-slab per rank with halo exchanges (strong scaling)")
    ap.add_argument("--layer-halo", action="store_true",
                    help="slab workload: exchange whole ghost layers and compute them (instead of face planes)")
    ap.add_argument("--slabs", type=int, default=1,
                    help="slab workload on one GPU: slabs held in one process (exchanged by device copies)")
    ap.add_argument("--solves", type=int, default=256, help="batch workload: number of solves")
    ap.add_argument("--batch-steps", type=int, default=300, help="batch workload: RK4 steps per solve")
    ap.add_argument("--requests", type=int, default=48, help="serve workload: number of requests")
    ap.add_argument("--rate", type=float, default=1.5, help="serve workload: Poisson arrival rate (1/s)")
    ap.add_argument("--preempt", action="store_true",
                    help="serve workload: the chosen form without and with preemptive admission (results compared "
                         "bit for bit, p50/p99 of both)")
    ap.add_argument("--serve-chosen-only", action="store_true",
                    help="serve workload: only the compensated FP32 served form (a longer stream), with every k-th "
                         "request re-solved alone in FP64 (50 of them) as the accuracy check")
    ap.add_argument("--config", default=None,
                    help="JSON file of option values (keys: the option names, e.g. {\"workload\": \"serve\", "
                         "\"rate\": 0.6}); options given on the command line take precedence")
    first, _ = ap.parse_known_args()
    if first.config:
        with open(first.config) as f:
            cfg = {k.replace("-", "_"): v for k, v in json.load(f).items()}
        known = {a.dest for a in ap._actions}
        bad = sorted(set(cfg) - known)
        if bad:
            ap.error(f"--config: unknown options {bad}")
        ap.set_defaults(**cfg)
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "batch":
        run_batch(args)
    elif args.workload == "serve":
        run_serve(args)
    elif args.workload == "slab":
        run_slab(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
