#!/usr/bin/env python
"""Generate tests/golden/golden.npz: small seeded input/output vectors of the 3D path.

The reference (Julia, with unvendored HexSBPSAT/HexMeshes) cannot run in this
environment, so these vectors come from the C++ Float64 oracle (oracle/) and are
regression pins: they freeze the oracle's outputs on seeded inputs so that a
change to the oracle or to the library shows up as a mismatch against committed
numbers, on machines that only have the fixture file.  Every case stores its
inputs as well as its outputs; the tests never regenerate inputs.

Cases (all Float64):
  gll_N{2..8}      GLL x, H, G on [0,1]
  curved_warped    wave3d_curved_rhs!, N=4, 2^3 warped elements (A=0.05), ADM
                   background, Sommerfeld faces, curvilinear split form, eps_KO=0.1
  curved_affine    wave3d_curved_rhs!, N=5, 2x3x2 affine elements, Dirichlet data
                   on all six sides, affine form, eps_KO=0
  sipg_c1          rhs_wave3d! on the 4^3 x n=6 standing wave (tau=20) and 10 RK4
                   steps with KO 0.1 at CFL 0.25, H-energy history
  strong_warped    wave_strong_rhs_mesh!, N=5, 2^3 warped elements, tag-7 faces, R=1
  evolve_n8        5 RK4 steps of the n=8 warped ADM pulse workload (2^3 elements)

Run from the repository root:  python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

from oracle import oracle as O  # noqa: E402
from conftest import load_package  # noqa: E402


def main(out=os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden.npz")):
    O.build()
    W = load_package().workloads
    g = {}
    for N in range(2, 9):
        x, H, G = O.gll_ops(N)
        g[f"gll_N{N}_x"], g[f"gll_N{N}_H"], g[f"gll_N{N}_G"] = x, H, G

    # curved_warped
    o = O.OracleMesh(4, (2, 2, 2), A=0.05, outer_tag=7)
    p = W.adm_params(5)
    co = o.background(2, p)
    x, y, z = o.coords()
    Phi = W.gaussian_field(x, y, z, *W.pulses(5, 2))
    Pi = 0.5 * W.standing_wave(x, y, z)
    Pd, Qd = o.rhs_curved(co, Phi, Pi, eps_ko=0.1, bc=O.make_bc([2] * 6), use_metric=True)
    g.update(curved_warped_params=p, curved_warped_Phi=Phi, curved_warped_Pi=Pi,
             curved_warped_Phidot=Pd, curved_warped_Pidot=Qd)

    # curved_affine
    o = O.OracleMesh(5, (2, 3, 2), A=0.0, outer_tag=0)
    p = W.adm_params(6)
    co = o.background(2, p)
    x, y, z = o.coords()
    Phi = W.gaussian_field(x, y, z, *W.pulses(6, 3))
    Pi = W.standing_wave(x, y, z)
    rng = np.random.default_rng(6)
    data = rng.standard_normal((5, o.nn)) * 0.1
    bc = O.make_bc([1] * 6, gPhi=data[0], gPi=data[1], gDx=data[2], gDy=data[3], gDz=data[4])
    Pd, Qd = o.rhs_curved(co, Phi, Pi, eps_ko=0.0, bc=bc, use_metric=False)
    g.update(curved_affine_params=p, curved_affine_Phi=Phi, curved_affine_Pi=Pi, curved_affine_bcdata=data,
             curved_affine_Phidot=Pd, curved_affine_Pidot=Qd)

    # sipg_c1
    o = O.OracleMesh(6, 4, outer_tag=0)
    x, y, z = o.coords()
    u0 = W.standing_wave(x, y, z)
    utt = o.rhs_sipg(u0, np.zeros_like(u0), tau=20.0)
    dt = 0.25 * o.min_spacing()
    u, v, E = o.evolve_sipg(u0, np.zeros_like(u0), dt, 10, tau=20.0, eps_ko=0.1, record_energy=True)
    g.update(sipg_c1_u0=u0, sipg_c1_utt=utt, sipg_c1_dt=np.array([dt]), sipg_c1_u10=u, sipg_c1_v10=v,
             sipg_c1_energy=E)

    # strong_warped
    o = O.OracleMesh(5, 2, A=0.05, outer_tag=7)
    x, y, z = o.coords()
    u = W.gaussian_field(x, y, z, *W.pulses(7, 2))
    ut = 0.3 * W.standing_wave(x, y, z)
    g.update(strong_warped_u=u, strong_warped_ut=ut, strong_warped_utt=o.rhs_strong(u, ut, R=1.0))

    # evolve_n8
    o = O.OracleMesh(8, 2, A=0.05, outer_tag=7)
    p = W.adm_params(3)
    co = o.background(2, p)
    x, y, z = o.coords()
    Phi = W.gaussian_field(x, y, z, *W.pulses(3, 8))
    Pi = np.zeros_like(Phi)
    dt = 0.2 * o.min_spacing() / W.max_speed(p)
    P5, Q5, E = o.evolve_curved(co, Phi, Pi, dt, 5, bc=O.make_bc([2] * 6), use_metric=True, record_energy=True)
    g.update(evolve_n8_params=p, evolve_n8_Phi0=Phi, evolve_n8_dt=np.array([dt]), evolve_n8_Phi5=P5,
             evolve_n8_Pi5=Q5, evolve_n8_energy=E)

    np.savez_compressed(out, **g)
    print(out, os.path.getsize(out), "bytes")


if __name__ == "__main__":
    main()
