"""Python host mirror of WaveToySecondOrder.jl's 3D API over the C ABI.

Each function below keeps the name, argument meaning and error behaviour of
the Julia function it stands in for (cited per function), with torch CUDA
tensors in place of CuArrays.  All numerics run in libwavetoy_b200.so; there is
no CPU path: without the built library or without a GPU every call raises.

Array conventions: a field is a flat tensor of N^3*Ne values in the reference's
(N,N,N,Ne) column-major order (i fastest), dtype float64 (plain form) or
float32 (FP32 form), on the context's device.
"""
from __future__ import annotations

import ctypes as C
import math
import os
from dataclasses import dataclass, field
from typing import Optional, Sequence

_HERE = os.path.dirname(os.path.abspath(__file__))
# WAVETOY_B200_LIB selects another build of the library, e.g. the bounds-check
# variant libwavetoy_b200_bc.so (build.py --bounds-check)
LIB_PATH = os.environ.get("WAVETOY_B200_LIB") or os.path.join(_HERE, "libwavetoy_b200.so")

WT_F64, WT_F32 = 0, 1
BC_DIRICHLET, BC_SOMMERFELD, BC_EXCISION, BC_FULL_DIRICHLET = 1, 2, 3, 4
FACE_SUBLUMINAL, FACE_OUTFLOW, FACE_INFLOW, FACE_SONIC = 1, 2, 3, 4
SOMMERFELD_BDRY_TAG = 7
EXCISION_BDRY_TAG = 8
BG_MINKOWSKI, BG_CONSTANT_SHIFT, BG_ADM_PERTURBED, BG_RADIAL_SHIFT = 0, 1, 2, 3
# time-dependent backgrounds from a spacetime metric (MetricBackground3D): params (A, d, t0)
BG_GAUGE_WAVE, BG_SINE_SHIFT = 4, 5
# fixed-step explicit Runge-Kutta methods (pick_integrator_first_order)
ERK_RK4, ERK_TSIT5 = 0, 1
ERK_MAX_STAGES = 16
IC_EIGENMODE_CARTESIAN, IC_GAUSSIANS, IC_OUTGOING_PULSE, IC_PLANE_WAVE, IC_EIGENMODE_RADIAL = 0, 1, 2, 3, 4
# precision forms of an FP32 mesh (n = 8 contractions): CUDA cores, split BF16 three-term / two-term
FP32_CUDA_CORES, FP32_BF16X3, FP32_BF16X2, FP32_COMPENSATED = 0, 1, 2, 3
# multi-patch mesh kinds (evolve3d mesh_kind :cubed_cube, :inflated_cube, :radial_shell)
MESH_CUBED_CUBE, MESH_INFLATED_CUBE, MESH_RADIAL_SHELL = 1, 2, 3
# prescribed 4-metrics of the fully second-order curved path
CURVED4_MINKOWSKI, CURVED4_GAUGE_WAVE = 0, 1

_ERRORS = {-1: "EINVAL", -2: "ECUDA", -3: "ENOMEM", -4: "ENOTSUP", -5: "ENONFINITE", -6: "ETIMEOUT"}

_BC_FROM_SYMBOL = {"dirichlet": BC_DIRICHLET, "sommerfeld": BC_SOMMERFELD, "excision": BC_EXCISION,
                   "full_dirichlet": BC_FULL_DIRICHLET}


class WaveToyError(RuntimeError):
    """Raised when the library returns an error status (ErrorException in the reference)."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"{_ERRORS.get(code, code)}: {msg}")
        self.code = code


class _MeshDesc(C.Structure):
    _fields_ = [("N", C.c_int), ("M", C.c_int * 3), ("x0", C.c_double), ("x1", C.c_double),
                ("warp_A", C.c_double), ("periodic", C.c_int), ("outer_tag", C.c_int), ("precision", C.c_int)]


class _PatchDesc(C.Structure):
    _fields_ = [("kind", C.c_int), ("N", C.c_int), ("M", C.c_int), ("p", C.c_double * 3), ("outer_tag", C.c_int),
                ("inner_tag", C.c_int), ("precision", C.c_int)]


class _BgDesc(C.Structure):
    _fields_ = [("kind", C.c_int), ("p", C.c_double * 16)]


class _BcDesc(C.Structure):
    _fields_ = [("kinds", C.c_int * 6), ("sigma", C.c_double), ("excision_tag", C.c_int),
                ("gPhi", C.c_void_p), ("gPi", C.c_void_p), ("gDx", C.c_void_p), ("gDy", C.c_void_p),
                ("gDz", C.c_void_p)]


SERVE_HRRN, SERVE_SJF, SERVE_FIFO = 0, 1, 2
SERVE_AUTO = -1
# wt_serve_status
REQ_WAITING, REQ_RUNNING, REQ_FINISHED, REQ_CANCELLED, REQ_PREEMPTED = 0, 1, 2, 3, 4
SERVE_MAX_IC = 128


class _ServeDesc(C.Structure):
    _fields_ = [("hbm_budget", C.c_double), ("tick", C.c_int), ("max_active", C.c_int), ("fill_nodes", C.c_longlong),
                ("order", C.c_int), ("precision", C.c_int), ("fp32_form", C.c_int), ("auto_fp32_max_steps", C.c_int),
                ("keep_results", C.c_int), ("rate_f64", C.c_double), ("rate_f32", C.c_double),
                ("preempt", C.c_int)]


class _ServeRequest(C.Structure):
    _fields_ = [("arrival", C.c_double), ("mesh", _MeshDesc), ("bg", _BgDesc), ("ic_kind", C.c_int), ("nic", C.c_int),
                ("ic", C.c_double * SERVE_MAX_IC), ("cfl", C.c_double), ("max_speed", C.c_double), ("steps", C.c_int),
                ("bc", _BcDesc)]


class _SolveDesc(C.Structure):
    _fields_ = [("mesh_kind", C.c_int), ("mesh", _MeshDesc), ("patch", _PatchDesc), ("precision", C.c_int),
                ("bg", _BgDesc), ("ic_kind", C.c_int), ("nic", C.c_int), ("ic", C.c_double * SERVE_MAX_IC),
                ("ic_exact", C.c_int), ("bc", _BcDesc), ("use_metric", C.c_int), ("eps_ko", C.c_double),
                ("t0", C.c_double), ("t1", C.c_double), ("nt", C.c_int), ("cfl", C.c_double),
                ("max_speed", C.c_double)]


class _SolveSlice(C.Structure):
    _fields_ = [("y", C.c_double), ("z", C.c_double), ("capacity", C.c_longlong), ("count", C.c_longlong),
                ("nodes", C.c_void_p), ("xs", C.c_void_p), ("Phi", C.c_void_p), ("Pi", C.c_void_p)]


class _SolveInfo(C.Structure):
    _fields_ = [("dt", C.c_double), ("dx", C.c_double), ("mu", C.c_double), ("steps", C.c_longlong)]


class _ServeResult(C.Structure):
    _fields_ = [("precision", C.c_int), ("nodes", C.c_longlong), ("steps", C.c_int), ("dt", C.c_double),
                ("arrival", C.c_double), ("admitted", C.c_double), ("finished", C.c_double)]


_lib = None


def library():
    """Load libwavetoy_b200.so (fails loudly when it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with "
                          "`python wavetoysecondorder.jl_b200/build.py` (nvcc, sm_100a)")
    L = C.CDLL(LIB_PATH)
    vp, pvp, i, d, ll = C.c_void_p, C.POINTER(C.c_void_p), C.c_int, C.c_double, C.c_longlong
    sig = {
        "wt_ctx_create": [i, pvp], "wt_ctx_destroy": [vp], "wt_ctx_synchronize": [vp],
        "wt_ctx_get_stream": [vp, pvp], "wt_ctx_set_stream": [vp, vp],
        "wt_ctx_launch_count": [vp, C.POINTER(ll)], "wt_ctx_nonfinite": [vp, C.POINTER(i)],
        "wt_ctx_selftest_wait": [vp, i, ll],
        "wt_ctx_memory": [vp, C.POINTER(ll), C.POINTER(ll), C.POINTER(ll)],
        "wt_build_flags": [C.POINTER(i)], "wt_ctx_bounds_status": [vp, C.POINTER(C.c_uint)],
        "wt_mesh_debug_set_table": [vp, i, ll, i, i],
        "wt_ctx_inject_alloc_failure": [vp, ll],
        "wt_mesh_create": [vp, C.POINTER(_MeshDesc), pvp],
        "wt_mesh_create_arrays": [vp, i, ll, vp, vp, vp, vp, vp, vp, i, pvp],
        "wt_mesh_create_patches": [vp, C.POINTER(_PatchDesc), pvp],
        "wt_patch_mesh_arrays": [C.POINTER(_PatchDesc), C.POINTER(ll), vp, vp, vp, vp, vp, vp],
        "wt_mesh_destroy": [vp], "wt_mesh_info": [vp, C.POINTER(i), C.POINTER(ll), C.POINTER(i)],
        "wt_mesh_get": [vp, C.c_char_p, vp], "wt_mesh_set_bdry": [vp, vp],
        "wt_mesh_min_spacing": [vp, C.POINTER(d)],
        "wt_background_set": [vp, vp, C.POINTER(_BgDesc), pvp], "wt_background_set_arrays": [vp, vp, vp, pvp],
        "wt_coef_get": [vp, vp], "wt_coef_destroy": [vp],
        "wt_coef_set_time": [vp, vp, d], "wt_coef_get_time": [vp, C.POINTER(d)],
        "wt_workspace_create": [vp, vp, pvp], "wt_workspace_destroy": [vp], "wt_workspace_mu": [vp, C.POINTER(d)],
        "wt_rhs_curved": [vp, vp, vp, vp, vp, vp, vp, d, C.POINTER(_BcDesc), i],
        "wt_rhs_curved_noalloc": [vp, vp, vp, vp, vp, vp, d, d, C.POINTER(_BcDesc), i],
        "wt_mesh_set_fp32_form": [vp, i],
        "wt_gather_nodes": [vp, vp, vp, vp, i, vp],
        "wt_snapshot_save": [vp, vp, vp, vp, d, C.c_char_p],
        "wt_snapshot_load": [vp, vp, vp, vp, C.POINTER(d), C.c_char_p],
        "wt_curved4_background": [vp, vp, i, vp, d, vp, vp],
        "wt_rhs_curved4": [vp, vp, vp, vp, vp, vp, vp, d, i, d],
        "wt_mesh_release_setup_geometry": [vp],
        "wt_batch_create": [vp, C.POINTER(vp)], "wt_batch_destroy": [vp],
        "wt_batch_add": [vp, vp, vp, vp, vp, d, C.POINTER(_BcDesc), C.POINTER(i)],
        "wt_batch_remove": [vp, i], "wt_batch_set_autotune": [vp, i], "wt_batch_set_variant": [vp, i, i],
        "wt_batch_step": [vp, i],
        "wt_batch_info": [vp, C.POINTER(i), C.POINTER(ll), C.POINTER(i)],
        "wt_batch_group_info": [vp, i, C.POINTER(i), C.POINTER(i), C.POINTER(i), C.POINTER(i), C.POINTER(ll)],
        "wt_apply_D": [vp, vp, vp, vp, i], "wt_ko_add": [vp, vp, vp, vp, d],
        "wt_gradient3d": [vp, vp, vp, vp, vp, vp], "wt_divergence3d": [vp, vp, vp, vp, vp, vp],
        "wt_rhs_sipg": [vp, vp, vp, vp, vp, C.POINTER(C.c_double * 6), d, d],
        "wt_rhs_strong": [vp, vp, vp, vp, vp, d, d], "wt_lap_strong_cons": [vp, vp, vp, vp, d, d],
        "wt_energy": [vp, vp, vp, vp, vp, i, C.POINTER(d)],
        "wt_energy_lapse": [vp, vp, vp, vp, vp, i, C.POINTER(d)], "wt_energy_sipg": [vp, vp, vp, vp, d, C.POINTER(d)],
        "wt_l2_diff": [vp, vp, vp, vp, i, C.POINTER(d)],
        "wt_step_rk4_curved": [vp, vp, vp, vp, vp, d, i, d, C.POINTER(_BcDesc), i],
        "wt_step_erk_curved": [vp, vp, vp, vp, vp, d, i, i, d, C.POINTER(_BcDesc), i],
        "wt_step_erk_curved_tableau": [vp, vp, vp, vp, vp, d, i, i, vp, vp, vp, d, C.POINTER(_BcDesc), i],
        "wt_erk_tableau": [i, C.POINTER(i), vp, vp, vp],
        "wt_step_rk4_sipg": [vp, vp, vp, vp, d, i, C.POINTER(C.c_double * 6), d, d, d],
        "wt_evolve_curved_host": [vp, vp, vp, vp, vp, d, i, i, d, C.POINTER(_BcDesc), i, vp],
        "wt_evolve_curved_host_f32": [vp, vp, vp, vp, vp, d, i, i, d, C.POINTER(_BcDesc), i, vp],
        "wt_initial_data": [vp, vp, i, vp, i, d, vp, vp],
        "wt_initial_state": [vp, vp, i, vp, i, d, vp, vp], "wt_state_set_f64": [vp, vp, vp, vp, vp, vp],
        "wt_gll_operators": [i, vp, vp, vp],
        "wt_ctx_profile": [vp, i], "wt_ctx_profile_read": [vp, C.POINTER(d * 3), C.POINTER(ll * 3)],
        "wt_mesh_create_slab": [vp, C.POINTER(_MeshDesc), i, i, pvp],
        "wt_rk4_stage_curved": [vp, vp, vp, vp, vp, d, i, i, C.POINTER(_BcDesc), i],
        "wt_halo_size": [vp, C.POINTER(ll)], "wt_halo_copy": [vp, vp, vp, i, i, vp, i],
        "wt_rk4_stage_curved_layers": [vp, vp, vp, vp, vp, d, i, i, i, i, C.POINTER(_BcDesc), i],
        "wt_halo_face_size": [vp, C.POINTER(ll)], "wt_halo_face_copy": [vp, vp, vp, i, i, i, vp, i],
        "wt_workspace_set_mu": [vp, d], "wt_workspace_set_fused": [vp, i],
        "wt_rk4_stage_curved_ko": [vp, vp, vp, vp, vp, d, i, d, C.POINTER(_BcDesc), i],
        "wt_halo_state_copy": [vp, vp, vp, vp, i, i, i, vp, i],
        "wt_serve_create": [vp, C.POINTER(_ServeDesc), pvp], "wt_serve_destroy": [vp],
        "wt_serve_submit": [vp, C.POINTER(_ServeRequest), C.POINTER(i)], "wt_serve_poll": [vp, C.POINTER(i)],
        "wt_serve_run": [vp], "wt_serve_get_result": [vp, i, C.POINTER(_ServeResult)],
        "wt_serve_result_state": [vp, i, vp, vp],
        "wt_serve_status": [vp, i, C.POINTER(i), C.POINTER(i), C.POINTER(i)], "wt_serve_cancel": [vp, i],
        "wt_serve_preempt": [vp, i],
        "wt_state_checkpoint_size": [vp, C.POINTER(ll)], "wt_state_checkpoint_save": [vp, vp, vp, vp, vp, ll],
        "wt_state_checkpoint_load": [vp, vp, vp, vp, vp, ll],
        "wt_solve_desc_check": [C.POINTER(_SolveDesc), C.c_char_p, i],
        "wt_solve_nodes": [C.POINTER(_SolveDesc), C.POINTER(ll)],
        "wt_solve_schedule": [d, d, i, d, i, vp, C.POINTER(d), vp],
        "wt_evolve3d": [vp, C.POINTER(_SolveDesc), vp, vp, vp, vp, vp, C.POINTER(_SolveSlice),
                        C.POINTER(_SolveInfo)],
        "wt_slice_select": [vp, ll, d, d, d, ll, vp, vp, C.POINTER(ll)],
        "wt_serve_info": [vp, C.POINTER(i), C.POINTER(i), C.POINTER(i), C.POINTER(d), C.POINTER(d)],
        "wt_serve_cost": [C.POINTER(_ServeDesc), C.POINTER(_ServeRequest), C.POINTER(d), C.POINTER(i)],
        "wt_serve_queue_order": [i, d, i, vp, vp, vp, vp],
        "wt_serve_preempt_choice": [C.POINTER(_ServeDesc), d, i, vp, vp, vp, vp, ll, i, d, vp, C.POINTER(i)],
    }
    for name, args in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = C.c_int
    L.wt_last_error.argtypes = [vp]
    L.wt_last_error.restype = C.c_char_p
    _lib = L
    return L


def _torch():
    import torch
    return torch


def _ptr(t):
    if t is None:
        return None
    if not t.is_cuda:
        raise ValueError("expected a CUDA tensor")
    if not t.is_contiguous():
        raise ValueError("expected a contiguous tensor")
    return C.c_void_p(t.data_ptr())


class Context:
    """One CUDA stream (the KernelAbstractions backend queue of the reference)."""

    def __init__(self, device: int = 0, use_torch_stream: bool = True):
        torch = _torch()
        if not torch.cuda.is_available():
            raise RuntimeError("wavetoy_b200 needs a CUDA device; there is no CPU fallback")
        self.device = device
        self.h = C.c_void_p()
        rc = library().wt_ctx_create(device, C.byref(self.h))
        if rc != 0:
            raise WaveToyError(rc, f"wt_ctx_create(device={device}) failed")
        self._children = []  # weak references to meshes / coefficients / workspaces
        if use_torch_stream:
            with torch.cuda.device(device):
                s = torch.cuda.current_stream(device).cuda_stream
            # torch's default stream is the legacy default stream (handle 0); name it
            # explicitly as cudaStreamLegacy (0x1) so launches are ordered with torch's
            # work and torch.cuda.Event timings bracket them
            library().wt_ctx_set_stream(self.h, C.c_void_p(s if s else 1))

    def _adopt(self, obj):
        import weakref
        self._children.append(weakref.ref(obj))

    def check(self, rc: int, what: str = ""):
        if rc != 0:
            msg = library().wt_last_error(self.h)
            raise WaveToyError(rc, (msg.decode() if msg else "") + (f" [{what}]" if what else ""))

    def synchronize(self):
        self.check(library().wt_ctx_synchronize(self.h))

    def launch_count(self) -> int:
        n = C.c_longlong()
        self.check(library().wt_ctx_launch_count(self.h, C.byref(n)))
        return n.value

    def profile(self, enable: bool = True):
        self.check(library().wt_ctx_profile(self.h, int(enable)))

    def profile_read(self):
        """((K1 ms, K1 launches), (K2 ms, K2 launches), (fused-stage ms, launches)) since the last read."""
        ms = (C.c_double * 3)()
        cnt = (C.c_longlong * 3)()
        self.check(library().wt_ctx_profile_read(self.h, C.byref(ms), C.byref(cnt)))
        return (ms[0], cnt[0]), (ms[1], cnt[1]), (ms[2], cnt[2])

    def selftest_wait(self, arrive: bool, polls: int = 1 << 16):
        """Run the bounded-wait self-test (wt_ctx_selftest_wait): raises WaveToyError
        (ETIMEOUT) when the wait gives up (arrive=False)."""
        self.check(library().wt_ctx_selftest_wait(self.h, int(bool(arrive)), int(polls)), "wt_ctx_selftest_wait")

    def nonfinite(self) -> bool:
        f = C.c_int()
        self.check(library().wt_ctx_nonfinite(self.h, C.byref(f)))
        return bool(f.value)

    def memory(self):
        """(live bytes, live allocations, allocations so far) of the device memory
        this context's objects hold."""
        v = [C.c_longlong() for _ in range(3)]
        self.check(library().wt_ctx_memory(self.h, *[C.byref(x) for x in v]))
        return tuple(x.value for x in v)

    def bounds_status(self) -> int:
        """Read and clear the bounds word of the bounds-check build (bit 0: an element index
        out of range, bit 1: a boundary slot); always 0 in the normal build."""
        w = C.c_uint()
        self.check(library().wt_ctx_bounds_status(self.h, C.byref(w)))
        return w.value

    def inject_alloc_failure(self, after: int):
        """Make the device allocation `after` allocations from now fail once with
        WT_ENOMEM (host side; after < 0 cancels)."""
        self.check(library().wt_ctx_inject_alloc_failure(self.h, int(after)))

    def close(self):
        """Destroy the context after every object made on it (children first:
        workspaces and coefficients, then meshes)."""
        if getattr(self, "h", None):
            alive = [r() for r in getattr(self, "_children", [])]
            for kind in (ServeEngine, Batch, Workspace, Coef, Mesh):
                for o in alive:
                    if isinstance(o, kind):
                        o.close()
            library().wt_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class _Child:
    def _ctx_alive(self) -> bool:
        c = self.ctx if hasattr(self, "ctx") else self.mesh.ctx
        return getattr(c, "h", None) is not None


class Mesh(_Child):
    """Mesh + MeshGeometry (+ metric terms) on the device.

    Stands in for HexMeshes.make_uniform_hex / make_warped_uniform_hex followed
    by HexSBPSAT.make_element, make_operators, make_geometry, to_device and
    make_metric_terms3d (src/evolve.jl:1174-1196)."""

    def __init__(self, ctx: Context, h, N: int, Ne: int, precision: int):
        self.ctx, self.h, self.N, self.Ne, self.precision = ctx, h, N, Ne, precision
        self.nn = N ** 3 * Ne
        ctx._adopt(self)
        self.dtype = _torch().float64 if precision == WT_F64 else _torch().float32

    @classmethod
    def uniform_hex(cls, ctx: Context, N: int, M, x0: float = 0.0, x1: float = 1.0, *, periodic: bool = False,
                    outer_tag: int = 0, warp_A: float = 0.0, precision: int = WT_F64) -> "Mesh":
        if isinstance(M, int):
            M = (M, M, M)
        d = _MeshDesc()
        d.N = N
        for a in range(3):
            d.M[a] = int(M[a])
        d.x0, d.x1, d.warp_A = float(x0), float(x1), float(warp_A)
        d.periodic, d.outer_tag, d.precision = int(periodic), int(outer_tag), int(precision)
        h = C.c_void_p()
        ctx.check(library().wt_mesh_create(ctx.h, C.byref(d), C.byref(h)), "wt_mesh_create")
        m = cls(ctx, h, N, M[0] * M[1] * M[2], precision)
        m.M, m.x0, m.x1, m.warp_A, m.periodic = tuple(M), x0, x1, warp_A, periodic
        return m

    @classmethod
    def slab(cls, ctx: Context, N: int, M, z0: int, nz: int, x0: float = 0.0, x1: float = 1.0, *,
             periodic: bool = False, outer_tag: int = 0, warp_A: float = 0.0, precision: int = WT_F64) -> "Mesh":
        """Element layers z0 .. z0 + nz - 1 of the analytic cube uniform_hex(N, M, ...) builds
        (wt_mesh_create_slab): the same geometry, metric terms and tags per element; z faces
        toward layers outside the slab are cuts (no neighbour, no tag)."""
        if isinstance(M, int):
            M = (M, M, M)
        d = _MeshDesc()
        d.N = N
        for a in range(3):
            d.M[a] = int(M[a])
        d.x0, d.x1, d.warp_A = float(x0), float(x1), float(warp_A)
        d.periodic, d.outer_tag, d.precision = int(periodic), int(outer_tag), int(precision)
        h = C.c_void_p()
        ctx.check(library().wt_mesh_create_slab(ctx.h, C.byref(d), int(z0), int(nz), C.byref(h)),
                  "wt_mesh_create_slab")
        m = cls(ctx, h, N, M[0] * M[1] * nz, precision)
        m.M, m.x0, m.x1, m.warp_A, m.periodic = (M[0], M[1], nz), x0, x1, warp_A, periodic
        m.z0, m.whole_M = int(z0), tuple(M)
        return m

    @classmethod
    def warped_uniform_hex(cls, ctx: Context, N: int, M, x0: float = 0.0, x1: float = 1.0, A: float = 0.05, *,
                           periodic: bool = False, outer_tag: int = 0, precision: int = WT_F64) -> "Mesh":
        return cls.uniform_hex(ctx, N, M, x0, x1, periodic=periodic, outer_tag=outer_tag, warp_A=A,
                               precision=precision)

    @classmethod
    def from_arrays(cls, ctx: Context, N: int, coords, jac, neighbour, neighbour_face, orientation, bdry,
                    precision: int = WT_F64) -> "Mesh":
        """MeshGeometry arrays (host numpy, Julia layout, 1-based connectivity) -> device mesh."""
        import numpy as np
        coords = np.ascontiguousarray(coords, dtype=np.float64)
        jac = np.ascontiguousarray(jac, dtype=np.float64)
        nb = np.ascontiguousarray(neighbour, dtype=np.int32)
        nf = np.ascontiguousarray(neighbour_face, dtype=np.int32)
        ori = np.ascontiguousarray(orientation, dtype=np.int8)
        bd = np.ascontiguousarray(bdry, dtype=np.int8)
        Ne = nb.size // 6
        h = C.c_void_p()
        ctx.check(library().wt_mesh_create_arrays(ctx.h, N, Ne, coords.ctypes.data, jac.ctypes.data,
                                                  nb.ctypes.data, nf.ctypes.data, ori.ctypes.data, bd.ctypes.data,
                                                  precision, C.byref(h)), "wt_mesh_create_arrays")
        return cls(ctx, h, N, Ne, precision)

    @classmethod
    def patches(cls, ctx: Context, kind: int, N: int, M: int, params: Sequence[float], *, outer_tag: int = 7,
                inner_tag: int = 8, precision: int = WT_F64) -> "Mesh":
        """Multi-patch curvilinear mesh: make_cubed_cube_mesh(T, M, R), make_inflated_cube_mesh(T, L, R1, R2, M)
        and make_radial_shell_mesh(T, R1, R2, M) as evolve3d builds them (src/evolve.jl:1176-1184), with this
        library's own patch maps; params = (R,), (L, R1, R2) or (R1, R2)."""
        d = _PatchDesc()
        d.kind, d.N, d.M = int(kind), int(N), int(M)
        for a, v in enumerate(list(params)[:3]):
            d.p[a] = float(v)
        d.outer_tag, d.inner_tag, d.precision = int(outer_tag), int(inner_tag), int(precision)
        h = C.c_void_p()
        ctx.check(library().wt_mesh_create_patches(ctx.h, C.byref(d), C.byref(h)), "wt_mesh_create_patches")
        ne = C.c_longlong()
        library().wt_mesh_info(h, None, C.byref(ne), None)
        m = cls(ctx, h, N, int(ne.value), precision)
        m.kind, m.M, m.params = kind, M, tuple(params)
        return m

    def get(self, name: str):
        import numpy as np
        n = self.nn
        sizes = {"coords": 3 * n, "jac": 9 * n, "invjac": 9 * n, "detjac": n, "Hphys": n, "Hd": n, "invdetJ": n,
                 "Ja": 9 * n, "x": self.N, "H": self.N, "G": self.N * self.N}
        isizes = {"bdry": 6 * self.Ne, "neighbour": 6 * self.Ne, "neighbour_face": 6 * self.Ne,
                  "orientation": 6 * self.Ne, "handedness": self.Ne}
        out = np.zeros(sizes[name]) if name in sizes else np.zeros(isizes[name], dtype=np.int32)
        self.ctx.check(library().wt_mesh_get(self.h, name.encode(), out.ctypes.data), f"wt_mesh_get({name})")
        return out

    def set_bdry(self, bdry):
        import numpy as np
        b = np.ascontiguousarray(bdry, dtype=np.int32)
        self.ctx.check(library().wt_mesh_set_bdry(self.h, b.ctypes.data), "wt_mesh_set_bdry")

    def release_setup_geometry(self):
        """Free the FP64 set-up geometry the RK4 path does not read (see wt_mesh_release_setup_geometry)."""
        self.ctx.check(library().wt_mesh_release_setup_geometry(self.h), "wt_mesh_release_setup_geometry")

    def set_fp32_form(self, form: int):
        """Select the precision form of an FP32 mesh (FP32_* constants; default FP32_COMPENSATED)."""
        self.ctx.check(library().wt_mesh_set_fp32_form(self.h, int(form)), "wt_mesh_set_fp32_form")

    def min_spacing(self) -> float:
        """_min_node_spacing_3d (src/evolve.jl:60-69)."""
        h = C.c_double()
        self.ctx.check(library().wt_mesh_min_spacing(self.h, C.byref(h)), "min_spacing")
        return h.value

    def empty(self, *shape):
        torch = _torch()
        return torch.empty(*(shape or (self.nn,)), dtype=self.dtype, device=f"cuda:{self.ctx.device}")

    def zeros(self):
        torch = _torch()
        return torch.zeros(self.nn, dtype=self.dtype, device=f"cuda:{self.ctx.device}")

    def close(self):
        if getattr(self, "h", None) and self._ctx_alive():
            library().wt_mesh_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Coef(_Child):
    """The coefficient bundle of make_coef3d / sample_background3d! (src/wave3d_curved.jl:106-124)."""

    def __init__(self, mesh: Mesh, h):
        self.mesh, self.h = mesh, h
        mesh.ctx._adopt(self)

    def get(self):
        """11 fields (alpha, sqrtg, b1, b2, b3, gu11, gu12, gu13, gu22, gu23, gu33), FP64 host."""
        import numpy as np
        out = np.zeros(11 * self.mesh.nn)
        self.mesh.ctx.check(library().wt_coef_get(self.h, out.ctypes.data), "wt_coef_get")
        return out

    def set_time(self, t: float):
        """Sample a time-dependent background (BG_GAUGE_WAVE, BG_SINE_SHIFT) at time t, as
        sample_background3d!(coef, bg, t) does for a MetricBackground3D."""
        self.mesh.ctx.check(library().wt_coef_set_time(self.mesh.ctx.h, self.h, float(t)), "wt_coef_set_time")

    @property
    def time(self) -> float:
        """The time a time-dependent background holds (RK4 stepping advances it); 0 for static ones."""
        t = C.c_double()
        library().wt_coef_get_time(self.h, C.byref(t))
        return float(t.value)

    def close(self):
        if getattr(self, "h", None) and self._ctx_alive():
            library().wt_coef_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def sample_background3d(mesh: Mesh, kind: int = BG_MINKOWSKI, params: Optional[Sequence[float]] = None) -> Coef:
    """make_coef3d + sample_background3d! for an analytic background (src/wave3d_curved.jl:106-124), or for a
    MetricBackground3D of the gauge wave / sine shift (kinds BG_GAUGE_WAVE, BG_SINE_SHIFT, params (A, d, t0)):
    time-dependent, re-sampled at every RK4 stage time by step_rk4_curved."""
    d = _BgDesc()
    d.kind = int(kind)
    params = () if params is None else list(params)
    if len(params) > len(d.p):
        raise ValueError(f"at most {len(d.p)} background parameters")
    for k, v in enumerate(params):
        d.p[k] = float(v)
    h = C.c_void_p()
    mesh.ctx.check(library().wt_background_set(mesh.ctx.h, mesh.h, C.byref(d), C.byref(h)), "wt_background_set")
    return Coef(mesh, h)


def background_from_arrays(mesh: Mesh, coef11) -> Coef:
    """Host-sampled 11-field bundle (the layout sample_background3d! fills)."""
    import numpy as np
    c = np.ascontiguousarray(coef11, dtype=np.float64)
    if c.size != 11 * mesh.nn:
        raise ValueError("coef11 must hold 11 fields of N^3*Ne values")
    h = C.c_void_p()
    mesh.ctx.check(library().wt_background_set_arrays(mesh.ctx.h, mesh.h, c.ctypes.data, C.byref(h)),
                   "wt_background_set_arrays")
    return Coef(mesh, h)


class Workspace(_Child):
    """Wave3DWorkspace: scratch + mu (src/wave3d_curved.jl:137-178)."""

    def __init__(self, mesh: Mesh):
        self.mesh, self.ctx = mesh, mesh.ctx
        self.h = C.c_void_p()
        self.ctx.check(library().wt_workspace_create(self.ctx.h, mesh.h, C.byref(self.h)), "wt_workspace_create")
        self.ctx._adopt(self)
        self._mu = None

    @property
    def mu(self) -> float:
        """Spectral-radius estimate of D_1^2 (30 power-iteration steps), computed on first use."""
        if self._mu is None:
            mu = C.c_double()
            self.ctx.check(library().wt_workspace_mu(self.h, C.byref(mu)), "wt_workspace_mu")
            self._mu = mu.value
        return self._mu

    def set_mu(self, mu: float):
        """Impose mu (wt_workspace_set_mu): the slabs of a partitioned solve take the whole mesh's."""
        self.ctx.check(library().wt_workspace_set_mu(self.h, float(mu)), "wt_workspace_set_mu")
        self._mu = float(mu)

    def set_fused(self, on: bool = True):
        """FP64 n = 8 RK4 steps through the fused stage kernel (wt_workspace_set_fused; the default)
        or through the two-kernel stages (on=False); the results are equal bit for bit."""
        self.ctx.check(library().wt_workspace_set_fused(self.h, int(bool(on))), "wt_workspace_set_fused")

    @property
    def inv_mu5(self) -> float:
        return (1.0 / self.mu) ** 5 if self.mu > 0 else 0.0

    def close(self):
        if getattr(self, "h", None) and self._ctx_alive():
            library().wt_workspace_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch(_Child):
    """Many independent solves advanced together (wt_batch_*; no counterpart in the
    reference, which runs one solve per evolve3d call).

    Members are (workspace, coefficients, Phi, Pi, dt, bc) sets on curvilinear
    meshes of any order and size.  Solves of one (n, precision, path) group run
    as one work list of (solve, element) tiles per kernel launch, one RK4 step
    of all groups is a CUDA graph, and the launch variant of the generic
    kernels (elements per CTA, or the pipelined kernels for n = 4, 6) is picked
    by timing when the membership changes."""

    def __init__(self, ctx: Context, autotune: bool = True):
        self.ctx = ctx
        self.h = C.c_void_p()
        ctx.check(library().wt_batch_create(ctx.h, C.byref(self.h)), "wt_batch_create")
        ctx._adopt(self)
        self._keep = {}
        if not autotune:
            ctx.check(library().wt_batch_set_autotune(self.h, 0), "wt_batch_set_autotune")

    def add(self, Phi, Pi, coef: "Coef", ws: "Workspace", dt: float, bc3d: Optional["BC3D"] = None) -> int:
        p, keep = _bcptr(bc3d)
        slot = C.c_int()
        self.ctx.check(library().wt_batch_add(self.h, ws.h, coef.h, _ptr(Phi), _ptr(Pi), float(dt), p,
                                              C.byref(slot)), "wt_batch_add")
        self._keep[slot.value] = (Phi, Pi, coef, ws, keep, p)
        return slot.value

    def remove(self, slot: int):
        self.ctx.check(library().wt_batch_remove(self.h, int(slot)), "wt_batch_remove")
        self._keep.pop(slot, None)

    def set_variant(self, k1: int = -1, k2: int = -1):
        """Fix the launch variants of the generic groups' K1 and K2 (wt_batch_set_variant): 0 / 1 the
        generic kernels at the default / alternative elements per CTA, 2 the pipelined kernels
        (n = 4, 6); -1 leaves the choice to the autotuner."""
        self.ctx.check(library().wt_batch_set_variant(self.h, int(k1), int(k2)), "wt_batch_set_variant")

    def step(self, nsteps: int = 1):
        self.ctx.check(library().wt_batch_step(self.h, int(nsteps)), "wt_batch_step")

    def info(self):
        ns, nn, ng = C.c_int(), C.c_longlong(), C.c_int()
        self.ctx.check(library().wt_batch_info(self.h, C.byref(ns), C.byref(nn), C.byref(ng)), "wt_batch_info")
        return ns.value, nn.value, ng.value

    def groups(self):
        """[(N, precision, n8_path, epb_variant, tiles)] per group."""
        out = []
        for g in range(self.info()[2]):
            v = [C.c_int() for _ in range(4)] + [C.c_longlong()]
            self.ctx.check(library().wt_batch_group_info(self.h, g, *[C.byref(x) for x in v]), "wt_batch_group_info")
            out.append(tuple(x.value for x in v))
        return out

    def close(self):
        if getattr(self, "h", None) and self._ctx_alive():
            library().wt_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def serve_desc(hbm_budget: float = 150e9, tick: int = 50, max_active: Optional[int] = None,
               fill_nodes: Optional[int] = 8_000_000, order: int = SERVE_HRRN, precision: int = WT_F32,
               fp32_form: int = FP32_COMPENSATED, auto_fp32_max_steps: int = 2000, keep_results: bool = False,
               rate_f64: float = 0.0, rate_f32: float = 0.0, preempt: bool = False) -> _ServeDesc:
    """wt_serve_desc: admission and stepping policy of a ServeEngine (None: no limit; preempt:
    preemptive admission of short requests, wt_serve_desc.preempt)."""
    d = _ServeDesc()
    d.hbm_budget = float(hbm_budget)
    d.tick = int(tick)
    d.max_active = 0 if max_active is None else int(max_active)
    d.fill_nodes = 0 if fill_nodes is None else int(fill_nodes)
    d.order, d.precision, d.fp32_form = int(order), int(precision), int(fp32_form)
    d.auto_fp32_max_steps = int(auto_fp32_max_steps)
    d.keep_results = int(bool(keep_results))
    d.rate_f64, d.rate_f32 = float(rate_f64), float(rate_f32)
    d.preempt = int(bool(preempt))
    return d


# ---- evolve3d in one call (wt_solve_desc, wt_evolve3d) ------------------------------
MESH_KINDS = {"cubical": 0, "cubed_cube": MESH_CUBED_CUBE, "inflated_cube": MESH_INFLATED_CUBE,
              "radial_shell": MESH_RADIAL_SHELL}
BG_KINDS = {"minkowski": BG_MINKOWSKI, "constant_shift": BG_CONSTANT_SHIFT, "adm_perturbed": BG_ADM_PERTURBED,
            "radial_shift": BG_RADIAL_SHIFT, "gauge_wave": BG_GAUGE_WAVE, "sine_shift": BG_SINE_SHIFT}
IC_KINDS = {"eigenmode_cartesian": IC_EIGENMODE_CARTESIAN, "gaussians": IC_GAUSSIANS,
            "outgoing_pulse": IC_OUTGOING_PULSE, "plane_wave": IC_PLANE_WAVE, "eigenmode_radial": IC_EIGENMODE_RADIAL}


def solve_desc(N: int = 4, M=8, *, T: int = WT_F64, mesh_kind: int = 0, x0: float = 0.0, x1: float = 1.0,
               warp_A: float = 0.0, periodic: bool = False, outer_tag: int = SOMMERFELD_BDRY_TAG,
               patch_params: Sequence[float] = (), inner_tag: int = 8, background: int = BG_MINKOWSKI,
               bg_params: Sequence[float] = (), ic: int = IC_GAUSSIANS, ic_params: Sequence[float] = (),
               ic_exact: bool = False, bc3d: Optional["BC3D"] = None, metric: bool = True, eps_KO: float = 0.0,
               t0: float = 0.0, t1: float = 1.0, Nt: int = 200, cfl: float = 0.1,
               max_speed: float = 1.0) -> _SolveDesc:
    """wt_solve_desc: the keywords of evolve3d(formulation = :conservative; T, N, M, mesh_kind,
    background, ic, bc, eps_KO, t0, t1, Nt, cfl) (src/evolve.jl:1149-1166) over this library's
    mesh, background and initial-data descriptors (defaults as the reference's: N = 4, M = 8,
    t1 = 1, Nt = 200, cfl = 1/10)."""
    d = _SolveDesc()
    d.mesh_kind, d.precision = int(mesh_kind), int(T)
    if d.mesh_kind == 0:
        Ms = (M, M, M) if isinstance(M, int) else tuple(M)
        d.mesh.N = int(N)
        for a in range(3):
            d.mesh.M[a] = int(Ms[a])
        d.mesh.x0, d.mesh.x1, d.mesh.warp_A = float(x0), float(x1), float(warp_A)
        d.mesh.periodic, d.mesh.outer_tag = int(bool(periodic)), 0 if periodic else int(outer_tag)
    else:
        if not isinstance(M, int) or len(patch_params) > 3:
            raise ValueError("patch meshes take one M and at most 3 parameters")
        d.patch.kind, d.patch.N, d.patch.M = int(mesh_kind), int(N), int(M)
        for k, v in enumerate(patch_params):
            d.patch.p[k] = float(v)
        d.patch.outer_tag, d.patch.inner_tag = int(outer_tag), int(inner_tag)
    if len(bg_params) > 16 or len(ic_params) > SERVE_MAX_IC:
        raise ValueError("too many background or initial-data parameters")
    d.bg.kind = int(background)
    for k, v in enumerate(bg_params):
        d.bg.p[k] = float(v)
    d.ic_kind, d.nic, d.ic_exact = int(ic), len(ic_params), int(bool(ic_exact))
    for k, v in enumerate(ic_params):
        d.ic[k] = float(v)
    if bc3d is not None:
        if any(g is not None for g in (bc3d.gPhi, bc3d.gPi, bc3d.gDx, bc3d.gDy, bc3d.gDz)):
            raise ValueError("evolve3d takes no boundary data fields")
        d.bc = bc3d.cstruct()
    d.use_metric, d.eps_ko = int(bool(metric)), float(eps_KO)
    d.t0, d.t1, d.nt, d.cfl, d.max_speed = float(t0), float(t1), int(Nt), float(cfl), float(max_speed)
    return d


def solve_config(cfg: dict) -> _SolveDesc:
    """A wt_solve_desc from a JSON-style dict: the keyword names of solve_desc; kinds may be
    given by name ("mesh_kind": "cubed_cube", "background": "adm_perturbed", "ic": "gaussians"),
    T as "Float64" / "Float32", the boundary as "bc": {"kinds": [...], "sigma": 1, "excision_tag": 0}."""
    kw = dict(cfg)
    for key, table in (("mesh_kind", MESH_KINDS), ("background", BG_KINDS), ("ic", IC_KINDS)):
        if isinstance(kw.get(key), str):
            if kw[key] not in table:
                raise ValueError(f"unknown {key} {kw[key]!r}: one of {sorted(table)}")
            kw[key] = table[kw[key]]
    if isinstance(kw.get("T"), str):
        kw["T"] = {"Float64": WT_F64, "Float32": WT_F32}[kw["T"]]
    if "bc" in kw:
        b = kw.pop("bc")
        kw["bc3d"] = make_bc3d(b["kinds"], sigma=b.get("sigma", 1.0), excision_tag=b.get("excision_tag", 0))
    if "M" in kw and isinstance(kw["M"], list):
        kw["M"] = tuple(kw["M"])
    return solve_desc(**kw)


def load_solve_config(path: str) -> _SolveDesc:
    """solve_config of a JSON file."""
    import json
    with open(path) as f:
        return solve_config(json.load(f))


def solve_desc_check(desc: _SolveDesc) -> str:
    """Why desc is not a valid solve ("" if it is); host only."""
    buf = C.create_string_buffer(256)
    library().wt_solve_desc_check(C.byref(desc), buf, 256)
    return buf.value.decode()


def solve_schedule(t0: float, t1: float, nt: int, dt: float, precision: int = WT_F64):
    """(steps before each sample, the last step's length, the sample times) of evolve3d's
    loop (wt_solve_schedule; host only)."""
    import numpy as np
    steps = np.zeros(max(int(nt), 1), dtype=np.int64)
    ts = np.zeros(max(int(nt), 1))
    last = C.c_double()
    rc = library().wt_solve_schedule(float(t0), float(t1), int(nt), float(dt), int(precision), steps.ctypes.data,
                                     C.byref(last), ts.ctypes.data)
    if rc != 0:
        raise WaveToyError(rc, "wt_solve_schedule: bad arguments")
    return steps, last.value, ts


def slice_select(xyz, y: float, z: float, atol: float):
    """The 1-D slice rule of evolve3d (_build_slice_3d, src/evolve.jl:104-123) on node-major
    coordinates (wt_slice_select; host only): (node indices, x) sorted by x."""
    import numpy as np
    xyz = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
    cnt = C.c_longlong()
    nodes = np.zeros(len(xyz), dtype=np.int64)
    xs = np.zeros(len(xyz))
    rc = library().wt_slice_select(xyz.ctypes.data, len(xyz), float(y), float(z), float(atol), len(xyz),
                                   nodes.ctypes.data, xs.ctypes.data, C.byref(cnt))
    if rc != 0:
        raise WaveToyError(rc, "wt_slice_select: bad arguments")
    return nodes[:cnt.value], xs[:cnt.value]


def evolve3d(ctx: Context, desc: _SolveDesc, slice_yz=(math.nan, math.nan), slice_capacity: int = 4096) -> dict:
    """evolve3d(formulation = :conservative; ...) (src/evolve.jl:1149-1366) in one call
    (wt_evolve3d): the sample times reached, energy and l2_err per sample, the 1-D slice
    (xs_line, Phis and Pis as [node, sample] like the reference's), the final state (host
    arrays of the solve's precision), dt, dx, mu and the steps taken.  slice_yz: the
    line (NaN: the mid-plane); slice_capacity: room for its nodes."""
    import numpy as np
    nn = C.c_longlong()
    if library().wt_solve_nodes(C.byref(desc), C.byref(nn)) != 0:
        raise WaveToyError(-1, "evolve3d: " + solve_desc_check(desc))
    dt_ = np.float64 if desc.precision == WT_F64 else np.float32
    Phi, Pi = np.empty(nn.value, dtype=dt_), np.empty(nn.value, dtype=dt_)
    ts, E, L = (np.empty(desc.nt) for _ in range(3))
    cap = int(slice_capacity)
    nodes, xs = np.zeros(cap, dtype=np.int64), np.zeros(cap)
    Ps, Qs = np.zeros((desc.nt, cap)), np.zeros((desc.nt, cap))
    sl = _SolveSlice(float(slice_yz[0]), float(slice_yz[1]), cap, 0, nodes.ctypes.data, xs.ctypes.data,
                     Ps.ctypes.data, Qs.ctypes.data)
    info = _SolveInfo()
    ctx.check(library().wt_evolve3d(ctx.h, C.byref(desc), Phi.ctypes.data, Pi.ctypes.data, ts.ctypes.data,
                                    E.ctypes.data, L.ctypes.data, C.byref(sl), C.byref(info)), "evolve3d")
    k = sl.count
    if k > cap:
        raise WaveToyError(-1, f"evolve3d: the slice has {k} nodes; raise slice_capacity")
    return {"ts_actual": ts, "energy": E, "l2_err": L, "xs_line": xs[:k], "slice_nodes": nodes[:k],
            "Phis": Ps[:, :k].T.copy(), "Pis": Qs[:, :k].T.copy(), "Phi_final": Phi, "Pi_final": Pi,
            "dt": info.dt, "dx": info.dx, "mu": info.mu, "steps": info.steps}


def serve_request(arrival: float, N: int, M, x0: float = 0.0, x1: float = 1.0, warp_A: float = 0.0,
                  outer_tag: int = 0, bg_kind: int = BG_MINKOWSKI, bg_params: Sequence[float] = (),
                  ic_kind: int = IC_GAUSSIANS, ic_params: Sequence[float] = (), cfl: float = 0.2,
                  max_speed: float = 1.0, steps: int = 1, bc3d: Optional["BC3D"] = None) -> _ServeRequest:
    """wt_serve_request: one solve (analytic mesh; background, a time-dependent one
    re-sampled at every RK4 stage; initial data of Phi with Pi = 0; dt = cfl * min
    spacing / max_speed; RK4 steps)."""
    q = _ServeRequest()
    q.arrival = float(arrival)
    M = (M, M, M) if isinstance(M, int) else tuple(M)
    q.mesh.N = int(N)
    for a in range(3):
        q.mesh.M[a] = int(M[a])
    q.mesh.x0, q.mesh.x1, q.mesh.warp_A = float(x0), float(x1), float(warp_A)
    q.mesh.periodic, q.mesh.outer_tag = 0, int(outer_tag)
    q.bg.kind = int(bg_kind)
    if len(bg_params) > len(q.bg.p) or len(ic_params) > SERVE_MAX_IC:
        raise ValueError("too many background or initial-data parameters")
    for k, v in enumerate(bg_params):
        q.bg.p[k] = float(v)
    q.ic_kind, q.nic = int(ic_kind), len(ic_params)
    for k, v in enumerate(ic_params):
        q.ic[k] = float(v)
    q.cfl, q.max_speed, q.steps = float(cfl), float(max_speed), int(steps)
    if bc3d is not None:
        if any(g is not None for g in (bc3d.gPhi, bc3d.gPi, bc3d.gDx, bc3d.gDy, bc3d.gDz)):
            raise ValueError("served requests take no boundary data fields")
        q.bc = bc3d.cstruct()
    return q


def serve_cost(desc: _ServeDesc, req: _ServeRequest):
    """(estimated device bytes, precision) of a request under a policy (wt_serve_cost; host only)."""
    b, p = C.c_double(), C.c_int()
    rc = library().wt_serve_cost(C.byref(desc), C.byref(req), C.byref(b), C.byref(p))
    if rc != 0:
        raise WaveToyError(rc, "wt_serve_cost: bad descriptor or request")
    return b.value, p.value


def serve_preempt_choice(desc: _ServeDesc, used: float, nodes, steps_left, cost, preemptions, head_nodes: int,
                         head_steps_left: int, head_cost: float):
    """The running requests (indices) that preemptive admission would preempt for the head request,
    in order (wt_serve_preempt_choice; host only)."""
    import numpy as np
    n = len(nodes)
    nodes = np.ascontiguousarray(nodes, dtype=np.int64)
    left = np.ascontiguousarray(steps_left, dtype=np.int32)
    cost = np.ascontiguousarray(cost, dtype=np.float64)
    pre = np.ascontiguousarray(preemptions, dtype=np.int32)
    out = np.zeros(max(n, 1), dtype=np.int32)
    cnt = C.c_int()
    rc = library().wt_serve_preempt_choice(C.byref(desc), float(used), n, nodes.ctypes.data, left.ctypes.data,
                                           cost.ctypes.data, pre.ctypes.data, int(head_nodes), int(head_steps_left),
                                           float(head_cost), out.ctypes.data, C.byref(cnt))
    if rc != 0:
        raise WaveToyError(rc, "wt_serve_preempt_choice: bad arguments")
    return [int(v) for v in out[:cnt.value]]


def serve_queue_order(order: int, now: float, arrival, service, work):
    """Admission order of waiting requests (wt_serve_queue_order; host only, no device)."""
    import numpy as np
    a = np.ascontiguousarray(arrival, dtype=np.float64)
    s = np.ascontiguousarray(service, dtype=np.float64)
    w = np.ascontiguousarray(work, dtype=np.float64)
    n = a.size
    if s.size != n or w.size != n:
        raise ValueError("arrival, service and work must have the same length")
    perm = np.zeros(n, dtype=np.int32)
    rc = library().wt_serve_queue_order(int(order), float(now), int(n), a.ctypes.data, s.ctypes.data, w.ctypes.data,
                                        perm.ctypes.data)
    if rc != 0:
        raise WaveToyError(rc, "wt_serve_queue_order: bad arguments")
    return perm.tolist()


class ServeEngine(_Child):
    """The native request server (wt_serve_*; no counterpart in the reference):
    requests arrive on the engine's clock (seconds since it was made), are
    admitted by the descriptor's order within the HBM budget, built on the
    device at admission and advanced together through one batch."""

    def __init__(self, ctx: Context, desc: _ServeDesc):
        self.ctx = ctx
        self.h = C.c_void_p()
        self.desc = desc
        ctx.check(library().wt_serve_create(ctx.h, C.byref(desc), C.byref(self.h)), "wt_serve_create")
        ctx._adopt(self)

    def submit(self, req: _ServeRequest) -> int:
        rid = C.c_int()
        self.ctx.check(library().wt_serve_submit(self.h, C.byref(req), C.byref(rid)), "wt_serve_submit")
        return rid.value

    def poll(self) -> int:
        n = C.c_int()
        self.ctx.check(library().wt_serve_poll(self.h, C.byref(n)), "wt_serve_poll")
        return n.value

    def run(self):
        self.ctx.check(library().wt_serve_run(self.h), "wt_serve_run")

    def result(self, rid: int) -> dict:
        r = _ServeResult()
        self.ctx.check(library().wt_serve_get_result(self.h, int(rid), C.byref(r)), "wt_serve_get_result")
        return {k: getattr(r, k) for k, _ in _ServeResult._fields_}

    def state(self, rid: int):
        """(Phi, Pi) device tensors holding a finished request's kept final state."""
        torch = _torch()
        r = self.result(rid)
        dt_ = torch.float64 if r["precision"] == WT_F64 else torch.float32
        Phi = torch.empty(r["nodes"], dtype=dt_, device=f"cuda:{self.ctx.device}")
        Pi = torch.empty_like(Phi)
        self.ctx.check(library().wt_serve_result_state(self.h, int(rid), _ptr(Phi), _ptr(Pi)), "wt_serve_result_state")
        return Phi, Pi

    def status(self, rid: int) -> dict:
        """{"status": REQ_*, "steps_left": ..., "preemptions": ...} of a request."""
        st, left, pre = C.c_int(), C.c_int(), C.c_int()
        self.ctx.check(library().wt_serve_status(self.h, int(rid), C.byref(st), C.byref(left), C.byref(pre)),
                       "wt_serve_status")
        return {"status": st.value, "steps_left": left.value, "preemptions": pre.value}

    def cancel(self, rid: int):
        self.ctx.check(library().wt_serve_cancel(self.h, int(rid)), "wt_serve_cancel")

    def preempt(self, rid: int):
        """Checkpoint a running request to host memory and put it back in the queue."""
        self.ctx.check(library().wt_serve_preempt(self.h, int(rid)), "wt_serve_preempt")

    def info(self) -> dict:
        w, a, dn, u, pk = C.c_int(), C.c_int(), C.c_int(), C.c_double(), C.c_double()
        self.ctx.check(library().wt_serve_info(self.h, C.byref(w), C.byref(a), C.byref(dn), C.byref(u), C.byref(pk)),
                       "wt_serve_info")
        return {"waiting": w.value, "active": a.value, "done": dn.value, "used_bytes": u.value,
                "peak_bytes": pk.value}

    def close(self):
        if getattr(self, "h", None) and self._ctx_alive():
            library().wt_serve_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def make_wave3d_workspace(mesh: Mesh) -> Workspace:
    """make_wave3d_workspace(geom, ops) (src/wave3d_curved.jl:158-178)."""
    return Workspace(mesh)


@dataclass
class BC3D:
    """make_bc3d bundle (src/boundaries3d.jl:45-52)."""
    kinds: tuple
    sigma: float = 1.0
    gPhi: object = None
    gPi: object = None
    gDx: object = None
    gDy: object = None
    gDz: object = None
    excision_tag: int = 0
    _c: object = field(default=None, repr=False)

    def cstruct(self) -> _BcDesc:
        b = _BcDesc()
        for f in range(6):
            b.kinds[f] = int(self.kinds[f])
        b.sigma = float(self.sigma)
        b.excision_tag = int(self.excision_tag)
        for nm in ("gPhi", "gPi", "gDx", "gDy", "gDz"):
            t = getattr(self, nm)
            setattr(b, nm, t.data_ptr() if t is not None else None)
        return b


def bc1d_kind(s) -> int:
    """bc1d_kind (src/boundaries1d.jl:73-77): Symbol -> BC_* code, ArgumentError otherwise."""
    if isinstance(s, int):
        return s
    key = str(s).lstrip(":")
    if key not in _BC_FROM_SYMBOL:
        raise ValueError(f"unknown 1D boundary condition {s} (expected :dirichlet, :sommerfeld, :excision, "
                         f":full_dirichlet)")
    return _BC_FROM_SYMBOL[key]


def make_bc3d(kinds, sigma: float = 1.0, gPhi=None, gPi=None, gDx=None, gDy=None, gDz=None,
              excision_tag: int = 0) -> BC3D:
    """make_bc3d(kinds; σ, gΦ, gΠ, gDx, gDy, gDz, excision_tag) (src/boundaries3d.jl:45-52)."""
    if len(kinds) != 6:
        raise ValueError("kinds must give one condition per face (-x,+x,-y,+y,-z,+z)")
    return BC3D(tuple(bc1d_kind(k) for k in kinds), sigma, gPhi, gPi, gDx, gDy, gDz, excision_tag)


def classify_face1d(a: float, beta: float, nhat: int, sonic_tol: Optional[float] = None) -> int:
    """classify_face1d (src/boundaries1d.jl:98-109)."""
    if sonic_tol is None:
        sonic_tol = 2.0 ** -13  # eps(Float64)^(1/4)
    s_R = a - beta
    s_L = -a - beta
    tol = sonic_tol * a
    if abs(s_R) <= tol or abs(s_L) <= tol:
        return FACE_SONIC
    out_R = s_R * nhat > 0
    out_L = s_L * nhat > 0
    if out_R and out_L:
        return FACE_OUTFLOW
    if not out_R and not out_L:
        return FACE_INFLOW
    return FACE_SUBLUMINAL


def classify_face3d(alpha, b1, b2, b3, gu11, gu22, gu33, naxis: int, nsign: int, sonic_tol=None) -> int:
    """classify_face3d (src/boundaries3d.jl:25-32); naxis is 1-based like the reference."""
    gunn = gu11 if naxis == 1 else gu22 if naxis == 2 else gu33
    bax = b1 if naxis == 1 else b2 if naxis == 2 else b3
    return classify_face1d(alpha * math.sqrt(gunn), bax, nsign, sonic_tol)


def validate_bc1d(cls: int, kind: int, face: str):
    """validate_bc1d (src/boundaries1d.jl:120-138): ArgumentError -> ValueError."""
    names = {FACE_SUBLUMINAL: "subluminal", FACE_OUTFLOW: "superluminal outflow",
             FACE_INFLOW: "superluminal inflow", FACE_SONIC: "sonic"}
    if cls == FACE_SONIC:
        raise ValueError(f"{face} boundary face is at a sonic point (|β| ≈ α/√γ): a characteristic speed "
                         "vanishes there and no boundary condition is well-posed")
    ok = ((cls == FACE_SUBLUMINAL and kind in (BC_DIRICHLET, BC_SOMMERFELD)) or
          (cls == FACE_OUTFLOW and kind == BC_EXCISION) or (cls == FACE_INFLOW and kind == BC_FULL_DIRICHLET))
    if not ok:
        raise ValueError(f"{face} boundary face is {names[cls]}; the boundary condition is not admissible")


def _bcptr(bc: Optional[BC3D]):
    if bc is None:
        return None, None
    s = bc.cstruct()
    return C.byref(s), s


def wave3d_curved_rhs(Phidot, Pidot, Phi, Pi, coef: Coef, ws: Workspace, eps_KO: float = 0.1,
                      bc3d: Optional[BC3D] = None, metric: bool = False):
    """wave3d_curved_rhs!(Φ̇, Π̇, Φ, Π, coef; geom, ops, ws, ε_KO, bc3d, metric) (src/wave3d_curved.jl:205-258).

    metric=True selects the curvilinear split-form path (the reference passes
    the metric-term bundle); False the affine per-axis path."""
    p, keep = _bcptr(bc3d)
    ws.ctx.check(library().wt_rhs_curved(ws.ctx.h, ws.h, coef.h, _ptr(Phi), _ptr(Pi), _ptr(Phidot), _ptr(Pidot),
                                         float(eps_KO), p, int(metric)), "wave3d_curved_rhs!")
    return Phidot, Pidot


NOALLOC_MAX_NODES = 262144
NOALLOC_MAX_BOUNDARY_NODES = 262144


def wave3d_curved_rhs_noalloc(Phidot, Pidot, Phi, Pi, coef: Coef, eps_KO: float = 0.0, mu: float = 0.0,
                              bc3d: Optional[BC3D] = None, metric: bool = False):
    """The RHS of wave3d_curved_rhs, with no workspace and no device allocation.

    For callers that may not allocate device memory while they evaluate the
    RHS (an embedding runtime that owns the device memory pool, a memory budget
    fixed before the time loop).  The scratch is a fixed device array of the
    library shared by all calls: meshes above NOALLOC_MAX_NODES nodes or
    NOALLOC_MAX_BOUNDARY_NODES boundary-face nodes raise WaveToyError (code
    WT_EINVAL), and calls
    that overlap on the GPU race.  mu (Workspace.mu of a workspace on the
    same mesh) is needed only when eps_KO != 0, and must then be positive and
    finite.  No counterpart in the reference."""
    p, keep = _bcptr(bc3d)
    ctx = coef.mesh.ctx
    ctx.check(library().wt_rhs_curved_noalloc(ctx.h, coef.h, _ptr(Phi), _ptr(Pi), _ptr(Phidot), _ptr(Pidot),
                                              float(eps_KO), float(mu), p, int(metric)), "wave3d_curved_rhs_noalloc")
    return Phidot, Pidot


def apply_D(Du, u, d: int, ws: Workspace):
    """HexSBPSAT.apply_D!(Du, u, d) (1-based axis d)."""
    ws.ctx.check(library().wt_apply_D(ws.ctx.h, ws.h, _ptr(u), _ptr(Du), int(d)), "apply_D!")
    return Du


def ko_add(dst, field_, eps_KO: float, ws: Workspace):
    """dst += ε μ⁻⁵ Σ_d D_d⁶ field (three _ko_axis3! calls, src/wave3d_curved.jl:182-192)."""
    ws.ctx.check(library().wt_ko_add(ws.ctx.h, ws.h, _ptr(dst), _ptr(field_), float(eps_KO)), "ko")
    return dst


def apply_gradient3d(g1, g2, g3, u, ws: Workspace):
    """apply_gradient3d!(DΦ1, DΦ2, DΦ3, Φ; geom, ops, metric) (src/wave3d_curved.jl:223)."""
    ws.ctx.check(library().wt_gradient3d(ws.ctx.h, ws.h, _ptr(u), _ptr(g1), _ptr(g2), _ptr(g3)), "gradient3d")
    return g1, g2, g3


def apply_divergence3d(out, F1, F2, F3, ws: Workspace):
    """apply_divergence3d!(Π̇, F1, F2, F3; geom, ops, metric) (src/wave3d_curved.jl:237)."""
    ws.ctx.check(library().wt_divergence3d(ws.ctx.h, ws.h, _ptr(F1), _ptr(F2), _ptr(F3), _ptr(out)),
                 "divergence3d")
    return out


def wave3d_energy(Phi, Pi, coef: Coef, ws: Workspace, metric: bool = False, lapse: bool = False) -> float:
    """wave3d_energy(Φ, Π, coef; geom, ops, ws, metric) (src/wave3d_curved.jl:268-287); lapse=True:
    the lapse-weighted energy (wt_energy_lapse), the norm conserved for a static background
    without shift when α != 1."""
    E = C.c_double()
    fn = library().wt_energy_lapse if lapse else library().wt_energy
    ws.ctx.check(fn(ws.ctx.h, ws.h, coef.h, _ptr(Phi), _ptr(Pi), int(metric), C.byref(E)), "wave3d_energy")
    return E.value


def _bv(bdry_values):
    arr = (C.c_double * 6)()
    for f in range(6):
        arr[f] = float(bdry_values[f])
    return arr


def rhs_wave3d(utt, u, ut, bdry_values, ws: Workspace, tau: float, sommerfeld_R: float = math.inf):
    """rhs_wave3d!(ü, u, u̇, bdry_values; geom, ops, work, τ, sommerfeld_R) (src/wave.jl:583-611)."""
    ws.ctx.check(library().wt_rhs_sipg(ws.ctx.h, ws.h, _ptr(u), _ptr(ut), _ptr(utt), C.byref(_bv(bdry_values)),
                                       float(tau), float(sommerfeld_R)), "rhs_wave3d!")
    return utt


def wave_strong_rhs_mesh(utt, u, ut, ws: Workspace, tau: Optional[float] = None, sommerfeld_R: float = math.inf):
    """wave_strong_rhs_mesh!(ü, u, u̇, mesh, geom, ops; τ = (N-1)², sommerfeld_R) (src/wave_strong_rhs.jl:296-360)."""
    if tau is None:
        tau = float((ws.mesh.N - 1) ** 2)
    ws.ctx.check(library().wt_rhs_strong(ws.ctx.h, ws.h, _ptr(u), _ptr(ut), _ptr(utt), float(tau),
                                         float(sommerfeld_R)), "wave_strong_rhs_mesh!")
    return utt


def wave_lap_strong_conservative_mesh(Lu, u, h: float, ws: Workspace, tau: Optional[float] = None):
    """wave_lap_strong_conservative_mesh!(Lu, u, mesh, ops, h; τ = (N-1)²) (src/wave_lap_strong.jl:280-308)."""
    if tau is None:
        tau = float((ws.mesh.N - 1) ** 2)
    ws.ctx.check(library().wt_lap_strong_cons(ws.ctx.h, ws.h, _ptr(u), _ptr(Lu), float(h), float(tau)),
                 "wave_lap_strong_conservative_mesh!")
    return Lu


def eval_curved_background(ginv, gam, mesh: Mesh, kind: int = CURVED4_MINKOWSKI, params=(0.0, 1.0), t: float = 0.0):
    """eval_curved_background!(ginv_all, Γc_all, mesh, xs, metric, t, h) (src/wave_curved_rhs.jl:373-418) for
    the analytic metrics CURVED4_MINKOWSKI and CURVED4_GAUGE_WAVE (params = (A, d)); ginv has 10 * nn and
    gam 4 * nn entries, component fastest."""
    p = (C.c_double * 2)(*[float(v) for v in list(params)[:2]])
    mesh.ctx.check(library().wt_curved4_background(mesh.ctx.h, mesh.h, int(kind), p, float(t), _ptr(ginv),
                                                   _ptr(gam)), "eval_curved_background!")
    return ginv, gam


def wave_curved_rhs_mesh(phidd, phi, phid, ginv, gam, ws: Workspace, h: float, conservative: bool = False,
                         tau: Optional[float] = None):
    """wave_curved_rhs_mesh! / wave_curved_rhs_conservative_mesh!(φ̈, φ, φ̇, mesh, ginv, Γc, ops, h; τ)
    (src/wave_curved_rhs.jl:155-362)."""
    if tau is None:
        tau = float((ws.mesh.N - 1) ** 2)
    ws.ctx.check(library().wt_rhs_curved4(ws.ctx.h, ws.h, _ptr(phi), _ptr(phid), _ptr(phidd), _ptr(ginv), _ptr(gam),
                                          float(h), int(conservative), float(tau)), "wave_curved_rhs_mesh!")
    return phidd


def energy_sipg(u, ut, ws: Workspace, tau: float) -> float:
    """½⟨u̇,u̇⟩_H − ½⟨u, L u⟩_H (test/kernels3d_tests.jl:39-47)."""
    E = C.c_double()
    ws.ctx.check(library().wt_energy_sipg(ws.ctx.h, ws.h, _ptr(u), _ptr(ut), float(tau), C.byref(E)), "energy")
    return E.value


def l2_diff(a, b, ws: Workspace, metric: bool = False) -> float:
    """sqrt(Σ (a−b)² H) (src/evolve.jl:1353-1354)."""
    out = C.c_double()
    ws.ctx.check(library().wt_l2_diff(ws.ctx.h, ws.h, _ptr(a), _ptr(b), int(metric), C.byref(out)), "l2")
    return out.value


def rk4_stage_curved(Phi, Pi, coef: Coef, ws: Workspace, dt: float, stage: int, part: int,
                     bc3d: Optional[BC3D] = None, metric: bool = False):
    """Part 1 (gradient, flux, Phi stage) or 2 (divergence, Pi stage) of RK4 stage 0..3 of
    step_rk4_curved with eps_KO = 0 (wt_rk4_stage_curved), for halo exchanges in between."""
    p, keep = _bcptr(bc3d)
    ws.ctx.check(library().wt_rk4_stage_curved(ws.ctx.h, ws.h, coef.h, _ptr(Phi), _ptr(Pi), float(dt), int(stage),
                                               int(part), p, int(bool(metric))), "wt_rk4_stage_curved")


def rk4_stage_curved_layers(Phi, Pi, coef: Coef, ws: Workspace, dt: float, stage: int, part: int, layer0: int,
                            nlayers: int, bc3d: Optional[BC3D] = None, metric: bool = False):
    """rk4_stage_curved on the element layers layer0 .. layer0 + nlayers - 1 only
    (wt_rk4_stage_curved_layers; analytic cubes and slabs)."""
    p, keep = _bcptr(bc3d)
    ws.ctx.check(library().wt_rk4_stage_curved_layers(ws.ctx.h, ws.h, coef.h, _ptr(Phi), _ptr(Pi), float(dt),
                                                      int(stage), int(part), int(layer0), int(nlayers), p,
                                                      int(bool(metric))), "wt_rk4_stage_curved_layers")


def halo_face_size(ws: Workspace) -> int:
    """Values of one packed face-plane halo (wt_halo_face_size; after a first stage part on ws)."""
    n = C.c_longlong()
    ws.ctx.check(library().wt_halo_face_size(ws.h, C.byref(n)), "wt_halo_face_size")
    return n.value


def halo_face_copy(ws: Workspace, Phi, stage: int, layer: int, face: int, buf, pack: bool):
    """Face `face` (4: -z, 5: +z) of element layer `layer`: the next stage's Phi and the three flux
    components on that face plane, into buf (pack) or back (wt_halo_face_copy)."""
    ws.ctx.check(library().wt_halo_face_copy(ws.ctx.h, ws.h, _ptr(Phi), int(stage), int(layer), int(face),
                                             _ptr(buf), int(bool(pack))), "wt_halo_face_copy")


def rk4_stage_curved_ko(Phi, Pi, coef: Coef, ws: Workspace, dt: float, stage: int, eps_KO: float,
                        bc3d: Optional[BC3D] = None, metric: bool = False):
    """One whole RK4 stage 0..3 of step_rk4_curved with Kreiss-Oliger dissipation eps_KO != 0
    (wt_rk4_stage_curved_ko), for halo exchanges between stages."""
    p, keep = _bcptr(bc3d)
    ws.ctx.check(library().wt_rk4_stage_curved_ko(ws.ctx.h, ws.h, coef.h, _ptr(Phi), _ptr(Pi), float(dt), int(stage),
                                                  float(eps_KO), p, int(bool(metric))), "wt_rk4_stage_curved_ko")


def halo_state_copy(ws: Workspace, Phi, Pi, stage: int, layer: int, count: int, buf, pack: bool):
    """count element layers from `layer` of the state the stage after `stage` reads (Phi's
    layers, then Pi's) into buf (pack) or back (wt_halo_state_copy)."""
    ws.ctx.check(library().wt_halo_state_copy(ws.ctx.h, ws.h, _ptr(Phi), _ptr(Pi), int(stage), int(layer), int(count),
                                              _ptr(buf), int(bool(pack))), "wt_halo_state_copy")


def halo_size(ws: Workspace) -> int:
    """Values of one packed halo layer (wt_halo_size; after a first stage part on ws)."""
    n = C.c_longlong()
    ws.ctx.check(library().wt_halo_size(ws.h, C.byref(n)), "wt_halo_size")
    return n.value


def halo_copy(ws: Workspace, Phi, stage: int, layer: int, buf, pack: bool):
    """Element layer `layer` of the fields read across faces after part 1 of `stage`
    (the next stage's Phi and the three flux components) into buf (pack) or back (wt_halo_copy)."""
    ws.ctx.check(library().wt_halo_copy(ws.ctx.h, ws.h, _ptr(Phi), int(stage), int(layer), _ptr(buf),
                                        int(bool(pack))), "wt_halo_copy")


def step_rk4_curved(Phi, Pi, coef: Coef, ws: Workspace, dt: float, nsteps: int, eps_KO: float = 0.0,
                    bc3d: Optional[BC3D] = None, metric: bool = False):
    """nsteps fixed-dt RK4 steps (OrdinaryDiffEq RK4(), adaptive=false; test/wave3d_tests.jl:32-44)."""
    p, keep = _bcptr(bc3d)
    ws.ctx.check(library().wt_step_rk4_curved(ws.ctx.h, ws.h, coef.h, _ptr(Phi), _ptr(Pi), float(dt), int(nsteps),
                                              float(eps_KO), p, int(metric)), "step_rk4_curved")
    return Phi, Pi


def step_erk_curved(Phi, Pi, coef: Coef, ws: Workspace, dt: float, nsteps: int, method: int = ERK_TSIT5,
                    eps_KO: float = 0.0, bc3d: Optional[BC3D] = None, metric: bool = False):
    """nsteps fixed-dt steps of the explicit RK method pick_integrator_first_order selects
    (src/evolve.jl:43-48; ERK_TSIT5 for N 5-6, ERK_RK4 for N <= 4), adaptive = false."""
    p, keep = _bcptr(bc3d)
    ws.ctx.check(library().wt_step_erk_curved(ws.ctx.h, ws.h, coef.h, _ptr(Phi), _ptr(Pi), float(dt), int(nsteps),
                                              int(method), float(eps_KO), p, int(metric)), "step_erk_curved")
    return Phi, Pi


def step_erk_curved_tableau(Phi, Pi, coef: Coef, ws: Workspace, dt: float, nsteps: int, c, A, b,
                            eps_KO: float = 0.0, bc3d: Optional[BC3D] = None, metric: bool = False):
    """nsteps fixed-dt steps of the caller's explicit Butcher tableau (c, A, b) with at most
    ERK_MAX_STAGES stages (wt_step_erk_curved_tableau), e.g. Vern7 with its published
    coefficients."""
    import numpy as np
    c = np.ascontiguousarray(c, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    A = np.ascontiguousarray(A, dtype=np.float64).reshape(len(c), len(c))
    p, keep = _bcptr(bc3d)
    ws.ctx.check(library().wt_step_erk_curved_tableau(ws.ctx.h, ws.h, coef.h, _ptr(Phi), _ptr(Pi), float(dt),
                                                      int(nsteps), len(c), c.ctypes.data, A.ctypes.data,
                                                      b.ctypes.data, float(eps_KO), p, int(metric)),
                 "step_erk_curved_tableau")
    return Phi, Pi


def composed_tableau(c, A, b, m: int):
    """The explicit tableau of m consecutive steps of (c, A, b), each of length dt / m, as one
    method with m s stages."""
    import numpy as np
    c, b, A = np.asarray(c, float), np.asarray(b, float), np.asarray(A, float).reshape(len(c), len(c))
    s = len(c)
    C2, B2, A2 = np.zeros(m * s), np.zeros(m * s), np.zeros((m * s, m * s))
    for p in range(m):
        C2[p * s:(p + 1) * s] = (p + c) / m
        B2[p * s:(p + 1) * s] = b / m
        A2[p * s:(p + 1) * s, p * s:(p + 1) * s] = A / m
        for q in range(p):
            A2[p * s:(p + 1) * s, q * s:(q + 1) * s] = b / m
    return C2, A2, B2


def erk_tableau(method: int):
    """(c, A, b) of the library's Butcher tableau for method (host only)."""
    import numpy as np
    st = C.c_int()
    if library().wt_erk_tableau(int(method), C.byref(st), None, None, None) != 0:
        raise WaveToyError(-1, f"unknown method {method}")
    n = st.value
    c, A, b = np.zeros(n), np.zeros(n * n), np.zeros(n)
    library().wt_erk_tableau(int(method), C.byref(st), c.ctypes.data, A.ctypes.data, b.ctypes.data)
    return c, A.reshape(n, n), b


def step_rk4_sipg(u, ut, ws: Workspace, dt: float, nsteps: int, bdry_values=(0,) * 6, tau: float = 20.0,
                  sommerfeld_R: float = math.inf, eps_KO: float = 0.0):
    """RK4 of the SIPG system (u, u̇) with optional KO on both."""
    ws.ctx.check(library().wt_step_rk4_sipg(ws.ctx.h, ws.h, _ptr(u), _ptr(ut), float(dt), int(nsteps),
                                            C.byref(_bv(bdry_values)), float(tau), float(sommerfeld_R),
                                            float(eps_KO)), "step_rk4_sipg")
    return u, ut


def gather_nodes(field, nodes, mesh: Mesh):
    """Values of a device field at the given node indices, as a float64 numpy array."""
    import numpy as np
    idx = np.ascontiguousarray(nodes, dtype=np.int64)
    out = np.zeros(len(idx))
    mesh.ctx.check(library().wt_gather_nodes(mesh.ctx.h, mesh.h, _ptr(field), idx.ctypes.data, len(idx),
                                             out.ctypes.data), "wt_gather_nodes")
    return out


def slice_nodes(mesh: Mesh, y_target: float, z_target: float, atol: float = 1.4901161193847656e-08):
    """The 1-D diagnostic slice of evolve3d (_build_slice_3d, src/evolve.jl:104-123): nodes with
    y, z strictly within atol of (y_target, z_target), the first node at each x (a node shared
    by two elements appears once), sorted by x (wt_slice_select).  Returns (node indices, x).
    Reads the set-up coordinates once."""
    return slice_select(mesh.get("coords"), y_target, z_target, atol)


def snapshot_save(path: str, Phi, Pi, mesh: Mesh, t: float = 0.0):
    """Write (Phi, Pi) and t to a snapshot file (64-byte header + raw fields)."""
    mesh.ctx.check(library().wt_snapshot_save(mesh.ctx.h, mesh.h, _ptr(Phi), _ptr(Pi), float(t),
                                              str(path).encode()), "wt_snapshot_save")


def snapshot_load(path: str, Phi, Pi, mesh: Mesh) -> float:
    """Read a snapshot written for a mesh of the same N, Ne and precision; returns t."""
    t = C.c_double()
    mesh.ctx.check(library().wt_snapshot_load(mesh.ctx.h, mesh.h, _ptr(Phi), _ptr(Pi), C.byref(t),
                                              str(path).encode()), "wt_snapshot_load")
    return t.value


def evolve_curved_device(Phi, Pi, coef: Coef, ws: Workspace, dt: float, steps_per_sample: int, nsamples: int,
                         eps_KO: float = 0.0, bc3d: Optional[BC3D] = None, metric: bool = False, slice_yz=None):
    """evolve3d's sample loop (src/evolve.jl:1339-1358) with the state kept on the device:
    per sample only the 1-D slice of Phi and Pi (slice_yz = (y, z), default the cube
    centre line), ||Phi||_H (zero reference) and the energy cross to the host.  Phi, Pi
    are device tensors advanced in place.  Returns dict(ts, xs_line, Phis, Pis, l2_err,
    energy) with time measured from the start."""
    import numpy as np
    mesh = ws.mesh
    if slice_yz is None:
        xyz = mesh.get("coords").reshape(-1, 3)
        slice_yz = (0.5 * (xyz[:, 1].min() + xyz[:, 1].max()), 0.5 * (xyz[:, 2].min() + xyz[:, 2].max()))
    nodes, xs = slice_nodes(mesh, *slice_yz)
    zero = mesh.zeros()
    Phis, Pis = np.zeros((len(nodes), nsamples)), np.zeros((len(nodes), nsamples))
    l2, E, ts = np.zeros(nsamples), np.zeros(nsamples), np.zeros(nsamples)
    for n in range(nsamples):
        step_rk4_curved(Phi, Pi, coef, ws, dt, steps_per_sample, eps_KO=eps_KO, bc3d=bc3d, metric=metric)
        ts[n] = (n + 1) * steps_per_sample * dt
        Phis[:, n] = gather_nodes(Phi, nodes, mesh)
        Pis[:, n] = gather_nodes(Pi, nodes, mesh)
        l2[n] = l2_diff(Phi, zero, ws, metric)
        E[n] = wave3d_energy(Phi, Pi, coef, ws, metric)
    if ws.ctx.nonfinite():
        raise WaveToyError(-5, "state became non-finite during evolution")
    return {"ts": ts, "xs_line": xs, "Phis": Phis, "Pis": Pis, "l2_err": l2, "energy": E}


def evolve_curved_host(Phi_host, Pi_host, coef: Coef, ws: Workspace, dt: float, steps_per_sample: int,
                       nsamples: int, eps_KO: float = 0.0, bc3d: Optional[BC3D] = None, metric: bool = False,
                       energy=None):
    """Host-buffer evolve in the shape of evolve3d(formulation = :conservative) (src/evolve.jl:1149-1366).

    Phi_host / Pi_host: C-contiguous host arrays in the mesh precision (float64
    numpy arrays or CPU torch tensors; page-locked torch tensors let the
    per-sample copies overlap the next sample's steps); they receive the final
    state.  energy: float64 array of length nsamples or None."""
    import numpy as np

    f32 = ws.mesh.precision == WT_F32

    def addr(a, want):
        if a is None:
            return None
        if hasattr(a, "data_ptr"):
            import torch
            if a.device.type != "cpu" or not a.is_contiguous() or a.dtype != getattr(torch, want):
                raise WaveToyError(-1, f"evolve_curved_host: expected a contiguous CPU {want} tensor")
            return C.c_void_p(a.data_ptr())
        if a.dtype != np.dtype(want) or not a.flags.c_contiguous:
            raise WaveToyError(-1, f"evolve_curved_host: expected a C-contiguous {want} array")
        return C.c_void_p(a.ctypes.data)

    sw = "float32" if f32 else "float64"
    fn = library().wt_evolve_curved_host_f32 if f32 else library().wt_evolve_curved_host
    p, keep = _bcptr(bc3d)
    ws.ctx.check(fn(ws.ctx.h, ws.h, coef.h, addr(Phi_host, sw), addr(Pi_host, sw), float(dt), int(steps_per_sample),
                    int(nsamples), float(eps_KO), p, int(metric), addr(energy, "float64")), "evolve_curved_host")


def patch_mesh_arrays(kind: int, N: int, M: int, params: Sequence[float], outer_tag: int = 7, inner_tag: int = 8):
    """Host arrays of a multi-patch mesh (the mesh Mesh.patches builds; no GPU needed): coords
    (3,N,N,N,Ne) and jac (9 per node) as flat float64, neighbour / neighbour_face (1-based, 0 = none),
    orientation (D4 code) and bdry as flat int32 of 6*Ne, in the reference's column-major order."""
    import numpy as np
    d = _PatchDesc()
    d.kind, d.N, d.M = int(kind), int(N), int(M)
    for a, v in enumerate(list(params)[:3]):
        d.p[a] = float(v)
    d.outer_tag, d.inner_tag, d.precision = int(outer_tag), int(inner_tag), WT_F64
    ne = C.c_longlong()
    rc = library().wt_patch_mesh_arrays(C.byref(d), C.byref(ne), None, None, None, None, None, None)
    if rc != 0:
        raise WaveToyError(rc, "wt_patch_mesh_arrays: bad mesh description")
    Ne, nn = int(ne.value), N ** 3 * int(ne.value)
    out = {"Ne": Ne, "coords": np.zeros(3 * nn), "jac": np.zeros(9 * nn)}
    for k in ("neighbour", "neighbour_face", "orientation", "bdry"):
        out[k] = np.zeros(6 * Ne, dtype=np.int32)
    rc = library().wt_patch_mesh_arrays(C.byref(d), C.byref(ne), out["coords"].ctypes.data, out["jac"].ctypes.data,
                                        *[out[k].ctypes.data for k in ("neighbour", "neighbour_face",
                                                                       "orientation", "bdry")])
    if rc != 0:
        raise WaveToyError(rc, "wt_patch_mesh_arrays failed")
    return out


def initial_data(mesh: Mesh, kind: int, params: Sequence[float], u, ut=None, t: float = 0.0):
    """Initial data / analytic references on the device: eigenmode_cartesian!,
    the :gaussian IC (summed pulses), outgoing_pulse!, the constant-shift plane
    wave and eigenmode_radial! (src/wave.jl:100-323, src/evolve.jl:1115-1118, 1257-1263)."""
    import numpy as np
    p = np.ascontiguousarray(params, dtype=np.float64)
    mesh.ctx.check(library().wt_initial_data(mesh.ctx.h, mesh.h, int(kind), p.ctypes.data if p.size else None,
                                             int(p.size), float(t), _ptr(u), _ptr(ut)), "initial_data")
    return u, ut


def initial_state(ws: "Workspace", kind: int, params: Sequence[float], Phi, Pi, t: float = 0.0):
    """initial_data of (Phi, Pi) = (u, u_t) for the solve ws steps, evaluated in FP64; on an FP32
    mesh the workspace keeps the low parts the FP32 arrays lose (wt_initial_state)."""
    import numpy as np
    p = np.ascontiguousarray(params, dtype=np.float64)
    ws.ctx.check(library().wt_initial_state(ws.ctx.h, ws.h, int(kind), p.ctypes.data if p.size else None,
                                            int(p.size), float(t), _ptr(Phi), _ptr(Pi)), "initial_state")
    return Phi, Pi


def state_from_f64(ws: "Workspace", Phi64, Pi64, Phi, Pi):
    """Load a Float64 device state into the state arrays ws steps (wt_state_set_f64): FP32 meshes keep
    the rounded values in Phi, Pi and the lost low parts in the workspace."""
    ws.ctx.check(library().wt_state_set_f64(ws.ctx.h, ws.h, _ptr(Phi64), _ptr(Pi64), _ptr(Phi), _ptr(Pi)),
                 "state_from_f64")
    return Phi, Pi


BUILD_BOUNDS_CHECK, BUILD_NVTX = 1, 2
TABLE_FACE_SOURCE, TABLE_BOUNDARY_SLOT = 0, 1


def build_flags() -> int:
    """BUILD_* bits of the loaded library (wt_build_flags)."""
    f = C.c_int()
    if library().wt_build_flags(C.byref(f)) != 0:
        raise WaveToyError(-1, "wt_build_flags")
    return f.value


def debug_set_table(mesh: "Mesh", table: int, e: int, f: int, value: int):
    """Overwrite entry (e, f) of a mesh's device face-source or boundary-slot table
    (bounds-check build only: wt_mesh_debug_set_table)."""
    mesh.ctx.check(library().wt_mesh_debug_set_table(mesh.h, int(table), int(e), int(f), int(value)),
                   "wt_mesh_debug_set_table")


def checkpoint_save(ws: "Workspace", Phi, Pi):
    """The stepped state (Phi, Pi) as a host checkpoint (numpy uint8), word for word, the FP32 low
    parts included (wt_state_checkpoint_save); synchronous."""
    import numpy as np
    n = C.c_longlong()
    ws.ctx.check(library().wt_state_checkpoint_size(ws.h, C.byref(n)), "wt_state_checkpoint_size")
    buf = np.empty(n.value, dtype=np.uint8)
    ws.ctx.check(library().wt_state_checkpoint_save(ws.ctx.h, ws.h, _ptr(Phi), _ptr(Pi), buf.ctypes.data, n.value),
                 "wt_state_checkpoint_save")
    return buf


def checkpoint_load(ws: "Workspace", Phi, Pi, buf):
    """Restore a checkpoint into the state arrays (Phi, Pi) that ws steps (wt_state_checkpoint_load)."""
    import numpy as np
    buf = np.ascontiguousarray(buf, dtype=np.uint8)
    ws.ctx.check(library().wt_state_checkpoint_load(ws.ctx.h, ws.h, _ptr(Phi), _ptr(Pi), buf.ctypes.data,
                                                    int(buf.size)), "wt_state_checkpoint_load")
    return Phi, Pi


def gaussian_params(centres, amps, widths):
    out = [float(len(amps))]
    for c, a, w in zip(centres, amps, widths):
        out += [float(c[0]), float(c[1]), float(c[2]), float(a), float(w)]
    return out


def gll_operators(N: int):
    """make_element + make_operators: GLL nodes x, SBP norm H and G (N x N) on [0,1]."""
    import numpy as np
    x = np.zeros(N); H = np.zeros(N); G = np.zeros(N * N)
    rc = library().wt_gll_operators(int(N), x.ctypes.data, H.ctypes.data, G.ctypes.data)
    if rc != 0:
        raise WaveToyError(rc, f"wt_gll_operators(N={N})")
    return x, H, G.reshape(N, N)
