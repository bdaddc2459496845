"""Serving loop for independent solves: requests arrive over time, their state
stays on the device, admission is bounded by an HBM budget, and admitted
solves advance together through one batch (wt_batch_*: the work-list kernels
over (solve, element) tiles and a CUDA graph per RK4 step), so requests that
arrive while others run join the work already on the GPU.  No counterpart in
the reference, whose evolve3d (src/evolve.jl:1149-1358) runs one solve per call.

A request is one warped-cube ADM solve (mesh size, order, background and
initial-data seeds, step count at CFL 0.2).  Latency = finish - arrival, where
finish is when its last step has completed on the device.
"""
from __future__ import annotations

import time
from collections import deque
from dataclasses import dataclass
from typing import List, Optional

from . import wavetoy as wt
from . import workloads as W


@dataclass
class Request:
    rid: int
    arrival: float          # seconds after the server starts
    elements: int           # elements per axis (cubic mesh)
    n: int                  # GLL nodes per axis
    steps: int              # RK4 steps
    seed: int
    scale: float = 1.0      # ADM perturbation scale (0: flat background)
    pulses: int = 2

    @staticmethod
    def from_dict(d) -> "Request":
        return Request(rid=d["rid"], arrival=d["arrival"], elements=d["elements"], n=d["n"], steps=d["steps"],
                       seed=d["seed"], scale=d.get("scale", 1.0), pulses=d.get("pulses", 2))

    @property
    def nodes(self) -> int:
        return self.elements ** 3 * self.n ** 3


@dataclass
class Result:
    rid: int
    arrival: float
    admitted: float
    finished: float
    nodes: int
    steps: int
    dt: float
    Phi: Optional[object] = None   # final state (device tensors) when keep_results
    Pi: Optional[object] = None

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


def request_dt(req: Request, mesh) -> float:
    """CFL 0.2 step of a request: 0.2 * dx_min / max_speed(background) (the
    speed bound sampled on 24^3 points)."""
    p = W.adm_params(req.seed, req.scale)
    return 0.2 * mesh.min_spacing() / W.max_speed(p, 24)


def build_solve(ctx, req: Request, precision: int, fp32_form: int = wt.FP32_CUDA_CORES, release: bool = True):
    """Mesh, background, workspace, initial data and dt of one request."""
    mesh = wt.Mesh.warped_uniform_hex(ctx, req.n, req.elements, 0.0, 1.0, 0.05, outer_tag=wt.SOMMERFELD_BDRY_TAG,
                                      precision=precision)
    if precision == wt.WT_F32:
        mesh.set_fp32_form(fp32_form)
    p = W.adm_params(req.seed, req.scale)
    coef = wt.sample_background3d(mesh, wt.BG_ADM_PERTURBED, p)
    ws = wt.make_wave3d_workspace(mesh)
    Phi, Pi = mesh.zeros(), mesh.zeros()
    c, a, w = W.pulses(req.seed, req.pulses, amp=(0.5, 1.0), width=(0.05, 0.15), centre=(0.25, 0.75))
    wt.initial_data(mesh, wt.IC_GAUSSIANS, wt.gaussian_params(c, a, w), Phi)
    dt = request_dt(req, mesh)
    if release:
        mesh.release_setup_geometry()
    return mesh, coef, ws, Phi, Pi, dt


def bytes_per_node(precision: int, n: int) -> int:
    """Device bytes one node of a served solve holds while it runs (set-up
    geometry released): coefficients, streamed metric, workspace and state;
    a little above the sum of the arrays, for the allocator's rounding."""
    if precision == wt.WT_F64:
        return 520 if n == 8 else 480
    return 300 if n == 8 else 260


# Precision policy of the "auto" form.  FP32 state with FP32-rounded
# coefficients perturbs the discrete operator by ~6e-8 relative, which shows
# up as a phase error that grows about linearly with the step count: measured
# on the served workload, 1e-5 relative L2 after 300-600 steps and up to 1e-4
# after 2000, the same for the split-BF16 tensor-core and the CUDA-core FP32
# forms.  Requests whose step count keeps the FP32 error under 1e-5 run in
# FP32, the others in FP64.
AUTO_FP32_MAX_STEPS = 250
AUTO = -1


def request_precision(precision: int, req: Request) -> int:
    if precision != AUTO:
        return precision
    return wt.WT_F32 if req.steps <= AUTO_FP32_MAX_STEPS else wt.WT_F64


class Server:
    """Continuous-batching server over one context (one GPU).  precision:
    wt.WT_F32, wt.WT_F64 or AUTO (per request, see request_precision); FP32 and
    FP64 requests share the batch (they run as separate groups)."""

    def __init__(self, ctx, precision: int = wt.WT_F32, hbm_budget: float = 150e9, tick: int = 50,
                 max_active: Optional[int] = None, fp32_form: int = wt.FP32_CUDA_CORES, keep_results: bool = False,
                 fill_nodes: Optional[int] = 8_000_000, order: str = "hrrn"):
        """fill_nodes: admit further requests only while the running ones hold fewer
        nodes than this (about what keeps the GPU busy); beyond it, new requests
        wait, so large requests are not slowed down by sharing the GPU with many
        others, while small ones still run together.  None: admit whatever the
        budget allows.  order: which waiting request is admitted next --
        "hrrn" (highest response ratio (wait + service) / service first, with the
        service time estimated from the request's DOF-updates: short requests go
        ahead under a backlog, and a long one's priority grows while it waits),
        "sjf" (least work first; long requests can wait until the backlog
        clears) or "fifo" (arrival order)."""
        if order not in ("hrrn", "sjf", "fifo"):
            raise ValueError("order must be 'hrrn', 'sjf' or 'fifo'")
        self.order = order
        self.ctx = ctx
        self.fill_nodes = fill_nodes
        self.precision = precision
        self.budget = float(hbm_budget)
        self.tick = int(tick)
        self.max_active = max_active
        self.fp32_form = fp32_form
        self.keep = keep_results

    def _service_s(self, req: Request) -> float:
        # rough service time at the measured single-GPU rates (FP64 ~3e9, FP32 ~6e9 DOF-updates/s)
        rate = 3e9 if request_precision(self.precision, req) == wt.WT_F64 else 6e9
        return 2.0 * req.nodes * req.steps / rate + 0.05

    def _cost(self, req: Request) -> float:
        # running footprint plus the FP64 set-up geometry held while it is built
        return req.nodes * (bytes_per_node(request_precision(self.precision, req), req.n) + 272)

    def run(self, requests: List[Request]) -> List[Result]:
        import torch
        batch = wt.Batch(self.ctx)
        pending = deque(sorted(requests, key=lambda r: r.arrival))
        for r in pending:
            if self._cost(r) > self.budget:
                raise ValueError(f"request {r.rid} ({r.nodes} nodes) does not fit the HBM budget")
        queue: deque = deque()
        active = {}
        used = 0.0
        self.peak_used = 0.0
        results: List[Result] = []
        t0 = time.perf_counter()
        while pending or queue or active:
            now = time.perf_counter() - t0
            while pending and pending[0].arrival <= now:
                queue.append(pending.popleft())
            if self.order == "sjf":
                queue = deque(sorted(queue, key=lambda r: (r.nodes * r.steps, r.arrival)))
            elif self.order == "hrrn":
                queue = deque(sorted(queue, key=lambda r: (-(now - r.arrival + self._service_s(r)) / self._service_s(r),
                                                           r.arrival)))
            # admit in queue order while the budget (and the slot limit) allows
            while queue and used + self._cost(queue[0]) <= self.budget and \
                    (self.max_active is None or len(active) < self.max_active) and \
                    (self.fill_nodes is None or not active or
                     sum(a["req"].nodes for a in active.values()) < self.fill_nodes):
                req = queue.popleft()
                used += self._cost(req)
                self.peak_used = max(self.peak_used, used)
                mesh, coef, ws, Phi, Pi, dt = build_solve(self.ctx, req, request_precision(self.precision, req),
                                                          self.fp32_form)
                slot = batch.add(Phi, Pi, coef, ws, dt, wt.make_bc3d([wt.BC_SOMMERFELD] * 6))
                active[slot] = {"req": req, "objs": (mesh, coef, ws), "Phi": Phi, "Pi": Pi, "dt": dt,
                                "left": req.steps, "admitted": time.perf_counter() - t0}
            if not active:
                if pending:
                    time.sleep(max(0.0, min(0.01, pending[0].arrival - (time.perf_counter() - t0))))
                continue
            k = min(self.tick, min(a["left"] for a in active.values()))
            batch.step(k)
            torch.cuda.synchronize(self.ctx.device)
            t_done = time.perf_counter() - t0
            for slot in [s for s, a in active.items() if a["left"] - k <= 0]:
                a = active.pop(slot)
                batch.remove(slot)
                req = a["req"]
                results.append(Result(req.rid, req.arrival, a["admitted"], t_done, req.nodes, req.steps, a["dt"],
                                      a["Phi"] if self.keep else None, a["Pi"] if self.keep else None))
                for o in reversed(a["objs"]):
                    o.close()
                used -= self._cost(req)
            for a in active.values():
                a["left"] -= k
        batch.close()
        if self.ctx.nonfinite():
            raise wt.WaveToyError(-5, "a served solve became non-finite")
        return sorted(results, key=lambda r: r.rid)


def percentile(values, q: float) -> float:
    import numpy as np
    return float(np.percentile(np.asarray(values, dtype=float), q)) if values else float("nan")


def summary(results: List[Result], makespan: float) -> dict:
    lat = [r.latency for r in results]
    dof = sum(2.0 * r.nodes * r.steps for r in results)
    return {"solves": len(results), "makespan_s": makespan, "solves_per_s": len(results) / makespan,
            "p50_latency_s": percentile(lat, 50), "p99_latency_s": percentile(lat, 99),
            "dof_updates_per_s": dof / makespan}
