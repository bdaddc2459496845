"""Serving loop for independent solves: requests arrive over time, their state
stays on the device, admission is bounded by an HBM budget, and admitted
solves advance together through one batch (wt_batch_*: the work-list kernels
over (solve, element) tiles and a CUDA graph per RK4 step), so requests that
arrive while others run join the work already on the GPU.  No counterpart in
the reference, whose evolve3d (src/evolve.jl:1149-1358) runs one solve per call.
The scheduling itself is native (wt_serve_*, wavetoy.ServeEngine); this module
describes requests, builds single solves for comparison and summarises runs.

A request is one warped-cube ADM solve (mesh size, order, background and
initial-data seeds, step count at CFL 0.2).  Latency = finish - arrival, where
finish is when its last step has completed on the device.
"""
from __future__ import annotations

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
    preemptions: int = 0           # times the request was preempted (preemptive admission)

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


def request_dt(req: Request, mesh) -> float:
    """CFL 0.2 step of a request: 0.2 * dx_min / max_speed(background) (the
    speed bound sampled on 24^3 points)."""
    p = W.adm_params(req.seed, req.scale)
    return 0.2 * mesh.min_spacing() / W.max_speed(p, 24)


def build_solve(ctx, req: Request, precision: int, fp32_form: int = wt.FP32_COMPENSATED, release: bool = True):
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
    wt.initial_state(ws, wt.IC_GAUSSIANS, wt.gaussian_params(c, a, w), Phi, Pi)
    dt = request_dt(req, mesh)
    if release:
        mesh.release_setup_geometry()
    return mesh, coef, ws, Phi, Pi, dt


# Precision policy of the "auto" form: requests of up to AUTO_FP32_MAX_STEPS
# steps run in the FP32 form the server is given, the others in FP64.  The
# plain FP32 forms (FP32_CUDA_CORES, FP32_BF16X3) lose Phi's FP32 rounding to
# the second derivative in Pi-dot and drift past 1e-5 relative L2 of the FP64
# result after 300-600 steps; the compensated form (the default) carries Phi's
# low part and differentiates it in FP64, and stays within 1e-5 over the
# workload's whole range of 200-2000 steps (tests/test_gpu_acceptance.py), so
# every request of the served workload runs in FP32.
AUTO_FP32_MAX_STEPS = 2000
AUTO = wt.SERVE_AUTO
ORDERS = {"hrrn": wt.SERVE_HRRN, "sjf": wt.SERVE_SJF, "fifo": wt.SERVE_FIFO}


def request_precision(precision: int, req: Request) -> int:
    if precision != AUTO:
        return precision
    return wt.WT_F32 if req.steps <= AUTO_FP32_MAX_STEPS else wt.WT_F64


def native_request(req: Request, with_speed: bool = True):
    """The wt_serve_request of a request: the warped cube of build_solve with its
    seeded ADM background and Gaussian pulses, CFL 0.2 (the speed bound sampled on
    24^3 points; with_speed=False leaves it 1, enough for the cost estimate)."""
    p = W.adm_params(req.seed, req.scale)
    c, a, w = W.pulses(req.seed, req.pulses, amp=(0.5, 1.0), width=(0.05, 0.15), centre=(0.25, 0.75))
    return wt.serve_request(req.arrival, req.n, req.elements, 0.0, 1.0, 0.05, outer_tag=wt.SOMMERFELD_BDRY_TAG,
                            bg_kind=wt.BG_ADM_PERTURBED, bg_params=p, ic_kind=wt.IC_GAUSSIANS,
                            ic_params=wt.gaussian_params(c, a, w), cfl=0.2,
                            max_speed=W.max_speed(p, 24) if with_speed else 1.0, steps=req.steps,
                            bc3d=wt.make_bc3d([wt.BC_SOMMERFELD] * 6))


class Server:
    """Continuous-batching server over one context (one GPU): the Python face of
    the native engine (wt_serve_*, wavetoy.ServeEngine), which does the
    admission, the device set-up of each admitted request and the batched
    stepping.  precision: wt.WT_F32, wt.WT_F64 or AUTO (per request, see
    request_precision); FP32 and FP64 requests share the batch (they run as
    separate groups)."""

    def __init__(self, ctx, precision: int = wt.WT_F32, hbm_budget: float = 150e9, tick: int = 50,
                 max_active: Optional[int] = None, fp32_form: int = wt.FP32_COMPENSATED, keep_results: bool = False,
                 fill_nodes: Optional[int] = 8_000_000, order: str = "hrrn", preempt: bool = False):
        """fill_nodes: admit further requests only while the running ones hold fewer
        nodes than this (about what keeps the GPU busy); beyond it, new requests
        wait, so large requests are not slowed down by sharing the GPU with many
        others, while small ones still run together.  None: admit whatever the
        budget allows.  order: which waiting request is admitted next --
        "hrrn" (highest response ratio (wait + service) / service first, with the
        service time estimated from the request's DOF-updates: short requests go
        ahead under a backlog, and a long one's priority grows while it waits),
        "sjf" (least work first; long requests can wait until the backlog
        clears) or "fifo" (arrival order).  preempt: preemptive admission -- a
        request that blocks a much shorter one is checkpointed to host memory and
        resumes later (wt_serve_desc.preempt)."""
        if order not in ORDERS:
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
        self.peak_used = 0.0
        self.preempt = bool(preempt)

    def desc(self):
        return wt.serve_desc(self.budget, self.tick, self.max_active, self.fill_nodes, ORDERS[self.order],
                             self.precision, self.fp32_form, AUTO_FP32_MAX_STEPS, self.keep, preempt=self.preempt)

    def _cost(self, req: Request) -> float:
        """Estimated device bytes of a request (the engine's own estimate)."""
        return wt.serve_cost(self.desc(), native_request(req, with_speed=False))[0]

    def run(self, requests: List[Request]) -> List[Result]:
        import torch
        for r in requests:
            if self._cost(r) > self.budget:
                raise ValueError(f"request {r.rid} ({r.nodes} nodes) does not fit the HBM budget")
        native = [(r, native_request(r)) for r in sorted(requests, key=lambda r: r.arrival)]
        eng = wt.ServeEngine(self.ctx, self.desc())   # its clock starts here
        try:
            rids = [(eng.submit(q), r) for r, q in native]
            eng.run()
            self.peak_used = eng.info()["peak_bytes"]
            results = []
            for rid, req in rids:
                x = eng.result(rid)
                Phi, Pi = eng.state(rid) if self.keep else (None, None)
                results.append(Result(req.rid, req.arrival, x["admitted"], x["finished"], x["nodes"], x["steps"],
                                      x["dt"], Phi, Pi, eng.status(rid)["preemptions"]))
            torch.cuda.synchronize(self.ctx.device)
        finally:
            eng.close()
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
