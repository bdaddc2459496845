"""ctypes front end of the CPU Float64 oracle (oracle/wavetoy_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, always as the checker.  The shipped library never
imports this module.

Array conventions follow the reference's Julia column-major layout: a field is
(N,N,N,Ne) with i fastest, stored here as a flat float64 numpy array of length
N^3*Ne (index i + N*(j + N*(k + N*e))).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SRC = os.path.join(_HERE, "wavetoy_oracle.cpp")
_LIB = os.path.join(_HERE, "_build", "liboracle.so")

BC_DIRICHLET, BC_SOMMERFELD, BC_EXCISION, BC_FULL_DIRICHLET = 1, 2, 3, 4


def build(force: bool = False) -> str:
    """Compile the oracle (g++ -O2 -fopenmp) into oracle/_build/liboracle.so."""
    os.makedirs(os.path.dirname(_LIB), exist_ok=True)
    if force or not os.path.exists(_LIB) or os.path.getmtime(_LIB) < os.path.getmtime(_SRC):
        subprocess.check_call(["g++", "-O2", "-fopenmp", "-fPIC", "-shared", "-o", _LIB, _SRC])
    return _LIB


class _BC(C.Structure):
    _fields_ = [("kinds", C.c_int32 * 6), ("sigma", C.c_double), ("excision_tag", C.c_int32),
                ("gPhi", C.c_void_p), ("gPi", C.c_void_p), ("gDx", C.c_void_p),
                ("gDy", C.c_void_p), ("gDz", C.c_void_p)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = C.CDLL(build())
        L = _lib
        vp, d, i = C.c_void_p, C.c_double, C.c_int
        L.or_mesh_create.restype = vp
        L.or_mesh_create.argtypes = [i, i, i, i, d, d, d, i, i]
        L.or_evolve_curved_td.argtypes = [vp, i, vp, vp, vp, d, i, d, C.POINTER(_BC), i]
        L.or_evolve_curved_erk.argtypes = [vp, vp, i, vp, vp, vp, d, i, i, d, C.POINTER(_BC), i]
        L.or_erk_tableau.argtypes = [i, vp, vp, vp]
        L.or_erk_tableau.restype = i
        L.or_mesh_create_arrays.restype = vp
        L.or_mesh_create_arrays.argtypes = [i, C.c_long, vp, vp, vp, vp, vp, vp]
        L.or_mesh_destroy.argtypes = [vp]
        L.or_mesh_ne.restype = C.c_long
        L.or_mesh_ne.argtypes = [vp]
        L.or_ops.argtypes = [i, vp, vp, vp]
        L.or_get.restype = i
        L.or_get.argtypes = [vp, C.c_char_p, vp]
        L.or_set_bdry.argtypes = [vp, vp]
        L.or_set.restype = i
        L.or_set.argtypes = [vp, C.c_char_p, vp]
        L.or_sample_background.argtypes = [vp, i, vp, vp]
        L.or_mu.restype = d
        L.or_mu.argtypes = [vp]
        L.or_apply_D.argtypes = [vp, vp, vp, i]
        L.or_grad3d.argtypes = [vp, vp, vp, vp, vp]
        L.or_div3d.argtypes = [vp, vp, vp, vp, vp]
        L.or_ko_add.argtypes = [vp, vp, vp, d]
        L.or_rhs_curved.argtypes = [vp, vp, vp, vp, vp, vp, d, C.POINTER(_BC), i, vp]
        L.or_energy.restype = d
        L.or_energy.argtypes = [vp, vp, vp, vp, i]
        L.or_energy_w.restype = d
        L.or_energy_w.argtypes = [vp, vp, vp, vp, i, i]
        L.or_rhs_sipg.argtypes = [vp, vp, vp, vp, vp, d, d]
        L.or_rhs_strong.argtypes = [vp, vp, vp, vp, d, d]
        L.or_lap_strong_cons.argtypes = [vp, vp, vp, d, d]
        L.or_rhs_curved4.argtypes = [vp, vp, vp, vp, vp, vp, d, i, d]
        L.or_curved4_background.argtypes = [vp, i, vp, d, vp, vp]
        L.or_evolve_curved.argtypes = [vp, vp, vp, vp, d, i, d, C.POINTER(_BC), i, vp]
        L.or_sipg_f.argtypes = [vp, vp, vp, vp, vp, vp, d, d, d]
        L.or_energy_sipg.restype = d
        L.or_energy_sipg.argtypes = [vp, vp, vp, d]
        L.or_evolve_sipg.argtypes = [vp, vp, vp, d, i, vp, d, d, d, vp]
        L.or_min_spacing.restype = d
        L.or_min_spacing.argtypes = [vp]
        L.or_num_threads.restype = i
    return _lib


def _p(a):
    if a is None:
        return None
    assert a.dtype in (np.float64, np.int32) and a.flags.c_contiguous
    return a.ctypes.data


def gll_ops(N: int):
    """GLL nodes x, weights H (diagonal of the SBP norm) and G on [0,1]."""
    x = np.zeros(N); H = np.zeros(N); G = np.zeros(N * N)
    lib().or_ops(N, _p(x), _p(H), _p(G))
    return x, H, G.reshape(N, N)


def make_bc(kinds, sigma=1.0, excision_tag=0, gPhi=None, gPi=None, gDx=None, gDy=None, gDz=None):
    """Boundary bundle mirroring make_bc3d (src/boundaries3d.jl:45-52)."""
    b = _BC()
    for f in range(6):
        b.kinds[f] = int(kinds[f])
    b.sigma = sigma
    b.excision_tag = excision_tag
    keep = []
    for name, arr in (("gPhi", gPhi), ("gPi", gPi), ("gDx", gDx), ("gDy", gDy), ("gDz", gDz)):
        if arr is not None:
            arr = np.ascontiguousarray(arr, dtype=np.float64)
            keep.append(arr)
            setattr(b, name, arr.ctypes.data)
    b._keep = keep
    return b


class OracleMesh:
    """Uniform / warped hex mesh with geometry and curl-form metric terms."""

    def __init__(self, N, M, x0=0.0, x1=1.0, A=0.0, periodic=False, outer_tag=0):
        if isinstance(M, int):
            M = (M, M, M)
        self.N = N
        self.M = tuple(M)
        self.h = lib().or_mesh_create(N, M[0], M[1], M[2], x0, x1, A, int(periodic), outer_tag)
        self.Ne = int(lib().or_mesh_ne(self.h))
        self.nn = N ** 3 * self.Ne
        self.x0, self.x1, self.A, self.periodic, self.outer_tag = x0, x1, A, periodic, outer_tag

    @classmethod
    def from_arrays(cls, N, coords, jac, nbr, nbrf, orient, bdry):
        """Mesh from arrays: coords (3*nn), jac (9*nn), 0-based topology (6*Ne: neighbour
        element or -1, neighbour face 0..5, orientation code, boundary tag)."""
        self = cls.__new__(cls)
        c = np.ascontiguousarray(coords, dtype=np.float64)
        J = np.ascontiguousarray(jac, dtype=np.float64)
        ti = [np.ascontiguousarray(a, dtype=np.int32) for a in (nbr, nbrf, orient, bdry)]
        Ne = ti[0].size // 6
        self.N, self.M = N, None
        self.h = lib().or_mesh_create_arrays(N, Ne, _p(c), _p(J), *[_p(a) for a in ti])
        self.Ne = int(lib().or_mesh_ne(self.h))
        self.nn = N ** 3 * self.Ne
        self.x0 = self.x1 = self.A = None
        self.periodic, self.outer_tag = False, None
        return self

    def __del__(self):
        try:
            if getattr(self, "h", None):
                lib().or_mesh_destroy(self.h)
        except Exception:
            pass

    def get(self, name):
        sizes = {"coords": 3 * self.nn, "jac": 9 * self.nn, "invjac": 9 * self.nn, "detjac": self.nn,
                 "Hphys": self.nn, "Ja": 9 * self.nn, "invdetJ": self.nn, "Hd": self.nn}
        isizes = {"nbr": 6 * self.Ne, "nbrf": 6 * self.Ne, "orient": 6 * self.Ne, "bdry": 6 * self.Ne,
                  "handed": self.Ne}
        if name in sizes:
            out = np.zeros(sizes[name])
        else:
            out = np.zeros(isizes[name], dtype=np.int32)
        rc = lib().or_get(self.h, name.encode(), _p(out))
        assert rc == 0, name
        return out

    def set_geometry(self, name, arr):
        arr = np.ascontiguousarray(arr, dtype=np.float64)
        assert lib().or_set(self.h, name.encode(), _p(arr)) == 0, name

    def set_bdry(self, bdry):
        bdry = np.ascontiguousarray(bdry, dtype=np.int32)
        lib().or_set_bdry(self.h, _p(bdry))

    def coords(self):
        c = self.get("coords").reshape(-1, 3)
        return c[:, 0].copy(), c[:, 1].copy(), c[:, 2].copy()

    def background(self, kind=0, params=None):
        p = np.zeros(16)
        if params is not None:
            p[: len(params)] = params
        coef = np.zeros(11 * self.nn)
        lib().or_sample_background(self.h, kind, _p(p), _p(coef))
        return coef

    def mu(self):
        return lib().or_mu(self.h)

    def apply_D(self, u, d):
        out = np.zeros(self.nn)
        lib().or_apply_D(self.h, _p(np.ascontiguousarray(u)), _p(out), d)
        return out

    def grad3d(self, u):
        g = [np.zeros(self.nn) for _ in range(3)]
        lib().or_grad3d(self.h, _p(np.ascontiguousarray(u)), _p(g[0]), _p(g[1]), _p(g[2]))
        return g

    def div3d(self, F1, F2, F3):
        out = np.zeros(self.nn)
        lib().or_div3d(self.h, _p(F1), _p(F2), _p(F3), _p(out))
        return out

    def ko_add(self, dst, field, koT):
        lib().or_ko_add(self.h, _p(dst), _p(field), koT)

    def rhs_curved(self, coef, Phi, Pi, eps_ko=0.0, bc=None, use_metric=False, want_grad=False):
        Phid = np.zeros(self.nn); Pid = np.zeros(self.nn)
        D = np.zeros(3 * self.nn) if want_grad else None
        lib().or_rhs_curved(self.h, _p(coef), _p(np.ascontiguousarray(Phi)), _p(np.ascontiguousarray(Pi)),
                            _p(Phid), _p(Pid), eps_ko, C.byref(bc) if bc is not None else None,
                            int(use_metric), _p(D))
        return (Phid, Pid, D) if want_grad else (Phid, Pid)

    def energy(self, coef, Phi, Pi, use_metric=False, lapse=False):
        """wave3d_energy; lapse=True: the alpha-weighted norm (see or_energy_w)."""
        return lib().or_energy_w(self.h, _p(coef), _p(np.ascontiguousarray(Phi)), _p(np.ascontiguousarray(Pi)),
                                 int(use_metric), int(bool(lapse)))

    def rhs_sipg(self, u, ut, bdry_values=(0,) * 6, tau=20.0, R=np.inf):
        out = np.zeros(self.nn)
        bv = np.asarray(bdry_values, dtype=np.float64)
        inv_R = 0.0 if not np.isfinite(R) else 1.0 / R
        lib().or_rhs_sipg(self.h, _p(np.ascontiguousarray(u)), _p(np.ascontiguousarray(ut)), _p(out), _p(bv),
                          tau, inv_R)
        return out

    def sipg_f(self, u, v, bdry_values=(0,) * 6, tau=20.0, R=np.inf, eps_ko=0.0):
        du = np.zeros(self.nn); dv = np.zeros(self.nn)
        bv = np.asarray(bdry_values, dtype=np.float64)
        inv_R = 0.0 if not np.isfinite(R) else 1.0 / R
        lib().or_sipg_f(self.h, _p(np.ascontiguousarray(u)), _p(np.ascontiguousarray(v)), _p(du), _p(dv),
                        _p(bv), tau, inv_R, eps_ko)
        return du, dv

    def energy_sipg(self, u, v, tau):
        return lib().or_energy_sipg(self.h, _p(np.ascontiguousarray(u)), _p(np.ascontiguousarray(v)), tau)

    def rhs_strong(self, u, ut, tau=None, R=np.inf):
        if tau is None:
            tau = float((self.N - 1) ** 2)
        out = np.zeros(self.nn)
        inv_R = 0.0 if not np.isfinite(R) else 1.0 / R
        lib().or_rhs_strong(self.h, _p(np.ascontiguousarray(u)), _p(np.ascontiguousarray(ut)), _p(out), tau,
                            inv_R)
        return out

    def lap_strong_cons(self, u, hel, tau=None):
        if tau is None:
            tau = float((self.N - 1) ** 2)
        out = np.zeros(self.nn)
        lib().or_lap_strong_cons(self.h, _p(np.ascontiguousarray(u)), _p(out), hel, tau)
        return out

    def curved4_background(self, kind=0, params=(0.0, 1.0), t=0.0):
        """eval_curved_background! (src/wave_curved_rhs.jl:373-418): kind 0 Minkowski,
        1 gauge wave (A, d).  Returns ginv (10*nn, component fastest) and gam (4*nn)."""
        ginv = np.zeros(10 * self.nn); gam = np.zeros(4 * self.nn)
        pp = np.asarray(list(params) + [0.0] * 2, dtype=np.float64)
        lib().or_curved4_background(self.h, int(kind), _p(pp), float(t), _p(ginv), _p(gam))
        return ginv, gam

    def rhs_curved4(self, phi, phid, ginv, gam, hel, conservative=False, tau=None):
        """wave_curved_rhs_mesh! / wave_curved_rhs_conservative_mesh! (src/wave_curved_rhs.jl:155-362)."""
        if tau is None:
            tau = float((self.N - 1) ** 2)
        out = np.zeros(self.nn)
        lib().or_rhs_curved4(self.h, _p(np.ascontiguousarray(phi, dtype=np.float64)),
                             _p(np.ascontiguousarray(phid, dtype=np.float64)), _p(out),
                             _p(np.ascontiguousarray(ginv, dtype=np.float64)),
                             _p(np.ascontiguousarray(gam, dtype=np.float64)), float(hel), int(conservative), tau)
        return out

    def evolve_curved(self, coef, Phi, Pi, dt, nsteps, eps_ko=0.0, bc=None, use_metric=False,
                      record_energy=False):
        Phi = np.array(Phi, dtype=np.float64, copy=True); Pi = np.array(Pi, dtype=np.float64, copy=True)
        E = np.zeros(nsteps + 1) if record_energy else None
        lib().or_evolve_curved(self.h, _p(coef), _p(Phi), _p(Pi), dt, nsteps, eps_ko,
                               C.byref(bc) if bc is not None else None, int(use_metric), _p(E))
        return (Phi, Pi, E) if record_energy else (Phi, Pi)

    def evolve_curved_td(self, kind, params, t0, Phi, Pi, dt, nsteps, eps_ko=0.0, bc=None, use_metric=False):
        """RK4 with the time-dependent background kind (4 gauge wave, 5 sine shift; params (A, d))
        re-sampled at every stage time from t0."""
        Phi = np.array(Phi, dtype=np.float64, copy=True); Pi = np.array(Pi, dtype=np.float64, copy=True)
        p = np.zeros(16)
        p[0], p[1], p[2] = params[0], params[1], t0
        lib().or_evolve_curved_td(self.h, int(kind), _p(p), _p(Phi), _p(Pi), dt, nsteps, eps_ko,
                                  C.byref(bc) if bc is not None else None, int(use_metric))
        return Phi, Pi

    def evolve_curved_erk(self, coef, Phi, Pi, dt, nsteps, method=1, eps_ko=0.0, bc=None, use_metric=False,
                          td=None):
        """Fixed-step explicit RK (method 1 Tsit5, 0 RK4) with the static coef, or with td =
        (kind, (A, d), t0) a time-dependent background re-sampled at every stage time."""
        Phi = np.array(Phi, dtype=np.float64, copy=True); Pi = np.array(Pi, dtype=np.float64, copy=True)
        p = np.zeros(16)
        kind = -1
        if td is not None:
            kind = int(td[0]); p[0], p[1], p[2] = td[1][0], td[1][1], td[2]
        lib().or_evolve_curved_erk(self.h, _p(coef) if coef is not None else None, kind, _p(p), _p(Phi), _p(Pi),
                                   dt, nsteps, int(method), eps_ko, C.byref(bc) if bc is not None else None,
                                   int(use_metric))
        return Phi, Pi

    def evolve_sipg(self, u, v, dt, nsteps, bdry_values=(0,) * 6, tau=20.0, R=np.inf, eps_ko=0.0,
                    record_energy=False):
        u = np.array(u, dtype=np.float64, copy=True); v = np.array(v, dtype=np.float64, copy=True)
        bv = np.asarray(bdry_values, dtype=np.float64)
        inv_R = 0.0 if not np.isfinite(R) else 1.0 / R
        E = np.zeros(nsteps + 1) if record_energy else None
        lib().or_evolve_sipg(self.h, _p(u), _p(v), dt, nsteps, _p(bv), tau, inv_R, eps_ko, _p(E))
        return (u, v, E) if record_energy else (u, v)

    def min_spacing(self):
        return lib().or_min_spacing(self.h)


# ---- initial data and analytic references (numpy, Float64) --------------------
# Restatements of the reference's closed-form fields, evaluated at node
# coordinates x, y, z; each returns (u, u_t).

def ic_eigenmode_cartesian(x, y, z, t, A, kx, ky, kz, om, x0, x1):
    """eigenmode_cartesian! (src/wave.jl:163-185)."""
    L = x1 - x0
    s = np.sin(kx * (x - x0) / L) * np.sin(ky * (y - x0) / L) * np.sin(kz * (z - x0) / L)
    return A * s * np.cos(om * t), -A * om * s * np.sin(om * t)


def ic_gaussians(x, y, z, pulses):
    """The :gaussian IC exp(-|x - c|^2 / (2 w^2)) (src/evolve.jl:1260-1263), one term per
    (cx, cy, cz, A, w) in pulses, scaled by A and summed; u_t = 0."""
    u = np.zeros_like(x)
    for cx, cy, cz, A, w in pulses:
        u = u + A * np.exp(-((x - cx) ** 2 + (y - cy) ** 2 + (z - cz) ** 2) / (2.0 * w * w))
    return u, np.zeros_like(x)


def _sinhc(v):
    """sinh(v)/v with the reference's Taylor branch for v^2 < 1/1000 (src/wave.jl:242-250)."""
    v = np.asarray(v, dtype=np.float64)
    v2 = v * v
    small = v2 < 1.0 / 1000.0
    safe = np.where(small, 1.0, v)
    return np.where(small, 1.0 + v2 * (1.0 / 6.0 + v2 * (1.0 / 120.0 + v2 * (1.0 / 5040.0))), np.sinh(safe) / safe)


def ic_outgoing_pulse(x, y, z, t, A, s0, sigma, cx, cy, cz):
    """outgoing_pulse! (src/wave.jl:292-323): u = 2A (b/s^2) sinhc(b r/s^2) exp(-(b^2 + r^2)/(2 s^2)),
    b = t + s0, and its time derivative."""
    is2 = 1.0 / (sigma * sigma)
    be = t + s0
    r2 = (x - cx) ** 2 + (y - cy) ** 2 + (z - cz) ** 2
    r = np.sqrt(r2)
    ex = np.exp(-0.5 * (be * be + r2) * is2)
    u = 2.0 * A * be * is2 * _sinhc(be * r * is2) * ex
    ut = -2.0 * A * is2 * ex * (be * be * is2 * _sinhc(be * r * is2) - np.cosh(be * r * is2))
    return u, ut


def ic_plane_wave(x, y, z, t, k, om, s):
    """Phi_e, Pi_e of _background3d :minkowski / :constant_shift (src/evolve.jl:1119-1120):
    Phi = sin(k (x + y + z) - om t), Pi = (-om - k s) cos(k (x + y + z) - om t)."""
    ph = k * (x + y + z) - om * t
    return np.sin(ph), (-om - k * s) * np.cos(ph)


def ic_eigenmode_radial(x, y, z, t, A, R, n, cx, cy, cz):
    """eigenmode_radial! (src/wave.jl:207-226): u = A sinc(n r / R) cos(om t), om = n pi / R,
    sinc(v) = sin(pi v)/(pi v)."""
    om = n * np.pi / R
    r = np.sqrt((x - cx) ** 2 + (y - cy) ** 2 + (z - cz) ** 2)
    sc = np.sinc(n * r / R)
    return A * sc * np.cos(om * t), -A * om * sc * np.sin(om * t)


def erk_tableau(method):
    """(c, A, b) of the oracle's Butcher tableau for method (1 Tsit5, 0 RK4)."""
    c, A, b = np.zeros(7), np.zeros(49), np.zeros(7)
    n = lib().or_erk_tableau(int(method), _p(c), _p(A), _p(b))
    return c[:n], A[: n * n].reshape(n, n), b[:n]


def num_threads() -> int:
    return lib().or_num_threads()
