"""Multi-patch curvilinear meshes (evolve3d's :cubed_cube, :inflated_cube,
:radial_shell, src/evolve.jl:1176-1184) and face orientation, on the CPU.

The builder's host arrays (wt_patch_mesh_arrays) are checked directly: faces
paired as neighbours coincide node for node under the stated orientation,
pairing is reciprocal, every Jacobian is positive and the quadrature volume is
the domain's.  The oracle, given the same arrays, passes the reference's
curvilinear tests (test/wave3d_tests.jl:109-142): a constant field is a steady
state of the RHS on all three meshes (free-stream) and the Sommerfeld spectrum
on the cubed cube is stable.  A warped uniform mesh whose elements' local axes
are turned by random rotations reaches every orientation code: its RHS is the
unturned mesh's RHS."""
import itertools

import numpy as np
import pytest

# the meshes of the reference's curvilinear RHS test (test/wave3d_tests.jl:111-114)
KINDS = [(1, 2, (0.3,)), (2, 1, (0.2, 0.5, 1.0)), (3, 2, (0.5, 1.0))]


def perm(ori, p, q, N):
    """The neighbour face point of (p, q) for orientation code ori (swap if bit 2,
    then reverse the first index if bit 0, the second if bit 1)."""
    a, b = (q, p) if ori & 4 else (p, q)
    return (N - 1 - a if ori & 1 else a), (N - 1 - b if ori & 2 else b)


def face_nodes(X, e, f, N):
    """X[e] is (N,N,N,3) indexed [k,j,i]; return the face's (p,q) -> coordinates grid [q,p,3]."""
    ax, r = f // 2, (N - 1 if f % 2 else 0)
    E = X[e]
    if ax == 0:
        return E[:, :, r, :]        # [k, j] = [q, p]
    if ax == 1:
        return E[:, r, :, :]        # [k, i] = [q, p]
    return E[r, :, :, :]            # [j, i] = [q, p]


def oracle_from(O, N, a):
    nb = a["neighbour"] - 1
    nf = np.where(a["neighbour"] > 0, a["neighbour_face"] - 1, 0)
    return O.OracleMesh.from_arrays(N, a["coords"], a["jac"], nb, nf, a["orientation"], a["bdry"])


@pytest.mark.parametrize("kind,M,p", KINDS)
def test_builder_faces_volume(wt, O, kind, M, p):
    N = 5
    a = wt.patch_mesh_arrays(kind, N, M, p)
    Ne = a["Ne"]
    X = a["coords"].reshape(Ne, N, N, N, 3)
    nb, nf, ori = a["neighbour"], a["neighbour_face"], a["orientation"]
    scale = np.abs(X).max()
    for i in range(6 * Ne):
        if nb[i] == 0:
            assert a["bdry"][i] != 0
            continue
        e, f, en, fn = i // 6, i % 6, nb[i] - 1, nf[i] - 1
        assert nb[fn + 6 * en] == e + 1 and nf[fn + 6 * en] == f + 1   # reciprocal
        A, B = face_nodes(X, e, f, N), face_nodes(X, en, fn, N)
        for q, pp in itertools.product(range(N), range(N)):
            pn, qn = perm(int(ori[i]), pp, q, N)
            assert np.abs(A[q, pp] - B[qn, pn]).max() < 1e-12 * scale
    J = a["jac"].reshape(-1, 3, 3)          # [node, b, a] = dX_a / dxi_b
    det = np.linalg.det(J)
    assert det.min() > 0
    _, H, _ = O.gll_ops(N)
    w = np.einsum("i,j,k->kji", H, H, H).ravel()
    vol = float(np.sum(np.tile(w, Ne) * det))
    want = 8.0 if kind == 1 else 4.0 / 3.0 * np.pi * (p[2] ** 3 if kind == 2 else p[1] ** 3 - p[0] ** 3)
    assert abs(vol - want) < (1e-12 if kind == 1 else 2e-3) * want
    if kind != 3:
        assert np.any(ori[nb > 0] != 0)     # mirrored patches meet with swapped face axes
    if kind == 3:
        assert set(np.unique(a["bdry"][nb == 0])) == {7, 8}


@pytest.mark.parametrize("kind,M,p", KINDS)
def test_oracle_free_stream(wt, O, kind, M, p):
    """A constant field is a steady state (test/wave3d_tests.jl:109-125), Sommerfeld
    outer faces, the radial shell's inner sphere excised (tag 8)."""
    N = 4
    o = oracle_from(O, N, wt.patch_mesh_arrays(kind, N, M, p))
    coef = o.background(0)
    Phi, Pi = np.full(o.nn, 2.5), np.zeros(o.nn)
    bc = O.make_bc([2] * 6, excision_tag=8)
    Pd, Qd = o.rhs_curved(coef, Phi, Pi, eps_ko=0.0, bc=bc, use_metric=True)
    assert np.abs(Pd).max() <= 1e-9 and np.abs(Qd).max() <= 1e-9


def test_oracle_cubed_cube_sommerfeld_spectrum(wt, O):
    """Curved Sommerfeld spectrum on the cubed cube with Kreiss-Oliger 0.1 is stable
    (test/wave3d_tests.jl:126-141)."""
    N = 4
    o = oracle_from(O, N, wt.patch_mesh_arrays(1, N, 1, (0.3,)))
    coef = o.background(0)
    bc = O.make_bc([2] * 6)
    nn = o.nn
    A = np.zeros((2 * nn, 2 * nn))
    for jc in range(2 * nn):
        u = np.zeros(2 * nn)
        u[jc] = 1.0
        Pd, Qd = o.rhs_curved(coef, u[:nn], u[nn:], eps_ko=0.1, bc=bc, use_metric=True)
        A[:nn, jc], A[nn:, jc] = Pd, Qd
    lam = np.linalg.eigvals(A)
    assert lam.real.max() <= 1e-5 * np.abs(lam).max()


def rotations():
    """The 24 proper rotations of the cube as (axis permutation, signs)."""
    out = []
    for pi in itertools.permutations(range(3)):
        par = 1 if sum(1 for i in range(3) for j in range(i + 1, 3) if pi[i] > pi[j]) % 2 == 0 else -1
        for s in itertools.product((1, -1), repeat=3):
            if par * s[0] * s[1] * s[2] == 1:
                out.append((pi, s))
    return out


def turned_mesh(O, base, N, seed):
    """Turn each element's local axes by a random rotation; returns the new arrays and,
    per element, the old local node of every new node."""
    rng = np.random.default_rng(seed)
    rots = rotations()
    Ne = base.Ne
    Xo = base.get("coords").reshape(Ne, N ** 3, 3)
    X = np.zeros_like(Xo)
    src = np.zeros((Ne, N ** 3), dtype=np.int64)
    for e in range(Ne):
        pi, s = rots[rng.integers(len(rots))] if e % 4 else rots[0]
        for k, j, i in itertools.product(range(N), repeat=3):
            t = (i, j, k)
            old = [t[pi[a]] if s[a] > 0 else N - 1 - t[pi[a]] for a in range(3)]
            src[e, i + N * (j + N * k)] = old[0] + N * (old[1] + N * old[2])
        X[e] = Xo[e, src[e]]
    _, _, G = O.gll_ops(N)
    Gm = np.asarray(G).reshape(N, N)
    Xg = X.reshape(Ne, N, N, N, 3)                      # [e, k, j, i, a]
    jac = np.zeros((Ne, N, N, N, 3, 3))                 # [..., b, a]
    jac[..., 0, :] = np.einsum("im,ekjma->ekjia", Gm, Xg)
    jac[..., 1, :] = np.einsum("jm,ekmia->ekjia", Gm, Xg)
    jac[..., 2, :] = np.einsum("km,emjia->ekjia", Gm, Xg)
    # topology by matching face centroids, orientation by matching face nodes
    Xf = X.reshape(Ne, N, N, N, 3)
    cen = np.array([[face_nodes(Xf, e, f, N)[[0, 0, -1, -1], [0, -1, 0, -1]].mean(0) for f in range(6)]
                    for e in range(Ne)])
    nb = np.zeros(6 * Ne, dtype=np.int32)
    nf = np.zeros(6 * Ne, dtype=np.int32)
    ori = np.zeros(6 * Ne, dtype=np.int32)
    bd = np.zeros(6 * Ne, dtype=np.int32)
    flat = cen.reshape(-1, 3)
    for i in range(6 * Ne):
        d = np.linalg.norm(flat - flat[i], axis=1)
        d[6 * (i // 6): 6 * (i // 6) + 6] = np.inf
        j = int(np.argmin(d))
        if d[j] > 1e-9:
            bd[i] = 7
            continue
        nb[i], nf[i] = j // 6 + 1, j % 6 + 1
        A, B = face_nodes(Xf, i // 6, i % 6, N), face_nodes(Xf, j // 6, j % 6, N)
        for c in range(8):
            if all(np.abs(A[q, pp] - B[perm(c, pp, q, N)[1], perm(c, pp, q, N)[0]]).max() < 1e-12
                   for q, pp in itertools.product(range(N), range(N))):
                ori[i] = c
                break
        else:
            raise AssertionError("faces do not coincide")
    return {"coords": X.ravel(), "jac": jac.ravel(), "neighbour": nb, "neighbour_face": nf, "orientation": ori,
            "bdry": bd}, src


def test_oracle_turned_elements_match(wt, O):
    """Every orientation code occurs, and the split-form RHS with its centred-flux SATs
    and Sommerfeld pass is that of the unturned mesh (Kreiss-Oliger off: apply_D!
    scales each local axis by its own diagonal Jacobian entry, which turning changes)."""
    N = 4
    base = O.OracleMesh(N, 3, A=0.05, outer_tag=7)
    arr, src = turned_mesh(O, base, N, 5)
    assert set(arr["orientation"][arr["neighbour"] > 0]) == set(range(8))
    # the unturned mesh through the same (discrete-Jacobian) path
    Ne = base.Ne
    Xo = base.get("coords")
    _, _, G = O.gll_ops(N)
    Gm = np.asarray(G).reshape(N, N)
    Xg = Xo.reshape(Ne, N, N, N, 3)
    jac0 = np.zeros((Ne, N, N, N, 3, 3))
    jac0[..., 0, :] = np.einsum("im,ekjma->ekjia", Gm, Xg)
    jac0[..., 1, :] = np.einsum("jm,ekmia->ekjia", Gm, Xg)
    jac0[..., 2, :] = np.einsum("km,emjia->ekjia", Gm, Xg)
    o0 = O.OracleMesh.from_arrays(N, Xo, jac0.ravel(), base.get("nbr"), base.get("nbrf"), base.get("orient"),
                                  base.get("bdry"))
    o1 = O.OracleMesh.from_arrays(N, arr["coords"], arr["jac"], arr["neighbour"] - 1,
                                  np.where(arr["neighbour"] > 0, arr["neighbour_face"] - 1, 0), arr["orientation"],
                                  arr["bdry"])
    p = wt.workloads.adm_params(2)
    rng = np.random.default_rng(8)
    x, y, z = o0.coords()
    Phi0 = np.sin(2 * x + y) * np.cos(3 * z) + 0.01 * rng.standard_normal(o0.nn)
    Pi0 = np.cos(x - 2 * y) * np.sin(z)
    gidx = (np.arange(Ne)[:, None] * N ** 3 + src).ravel()   # new node -> old node
    bc = O.make_bc([2] * 6)
    P0, Q0 = o0.rhs_curved(o0.background(2, p), Phi0, Pi0, eps_ko=0.0, bc=bc, use_metric=True)
    P1, Q1 = o1.rhs_curved(o1.background(2, p), Phi0[gidx], Pi0[gidx], eps_ko=0.0, bc=bc, use_metric=True)
    for a, b in ((P1, P0[gidx]), (Q1, Q0[gidx])):
        assert np.linalg.norm(a - b) <= 1e-11 * np.linalg.norm(b)


def test_oracle_radial_shell_excision_drains_noise(wt, O):
    """The reference's radial-shell excision check (test/evolve3d_curv_tests.jl:46-60): flat
    space with a radial shift ramping from V = 2 at R1 = 0.5 (superluminal: the inner sphere
    is excised, tag 8) to 1/20 at R2 = 1 (Sommerfeld), sqrt(eps) noise, eps_KO = 0.1, CFL 1/10
    with max speed V + 1, to t = 1: the energy never grows (here at every RK4 step, not only at
    the samples) and the noise drains out."""
    N, M, V = 4, 2, 2.0
    a = wt.patch_mesh_arrays(wt.MESH_RADIAL_SHELL, N, M, (0.5, 1.0))
    o = oracle_from(O, N, a)
    assert sorted(set(a["bdry"].tolist())) == [0, 7, 8]
    co = o.background(3, [V, 1.0 / 20, 0.5, 1.0])
    rng = np.random.default_rng(20260604)
    amp = np.sqrt(np.finfo(float).eps)
    P0, Q0 = amp * rng.standard_normal(o.nn), amp * rng.standard_normal(o.nn)
    dt = min(0.1 * o.min_spacing() / (V + 1), 1.4 / (0.1 * o.mu()))
    P, Q, E = o.evolve_curved(co, P0, Q0, dt, int(np.ceil(1.0 / dt)), eps_ko=0.1,
                              bc=O.make_bc([2] * 6, excision_tag=8), use_metric=True, record_energy=True)
    assert np.all(np.isfinite(P)) and np.all(np.isfinite(Q))
    assert np.all(np.diff(E) <= 1e-6 * E[0])
    assert E[-1] < 0.5 * E[0]


def test_oracle_cubed_cube_sommerfeld_noise_energy(wt, O):
    """The reference's cubed-cube Sommerfeld check (test/evolve3d_curv_tests.jl:36-44): N = 4,
    M = 1, R = 0.3, Minkowski, sqrt(eps) noise, eps_KO = 0.1, CFL 1/10, to t = 0.5: the energy
    never exceeds its start by more than 1e-6 (checked at every RK4 step)."""
    N = 4
    a = wt.patch_mesh_arrays(wt.MESH_CUBED_CUBE, N, 1, (0.3,))
    o = oracle_from(O, N, a)
    co = o.background(0)
    rng = np.random.default_rng(20260604)
    amp = np.sqrt(np.finfo(float).eps)
    P0, Q0 = amp * rng.standard_normal(o.nn), amp * rng.standard_normal(o.nn)
    dt = min(0.1 * o.min_spacing(), 1.4 / (0.1 * o.mu()))
    P, Q, E = o.evolve_curved(co, P0, Q0, dt, int(np.ceil(0.5 / dt)), eps_ko=0.1, bc=O.make_bc([2] * 6),
                              use_metric=True, record_energy=True)
    assert np.all(np.isfinite(P)) and np.all(np.isfinite(Q))
    assert E.max() <= E[0] * (1 + 1e-6)


@pytest.mark.parametrize("noise", [False, True])
def test_oracle_strong_form_inflated_cube_stays_bounded(wt, O, noise):
    """The reference's strong-form (full chain rule) checks on the inflated cube
    (test/wave_strong_rhs_tests.jl:89-151): N = 3, M = 4, L = 0.1, R1 = 0.3, R2 = 1, an outgoing
    pulse (A = 1, s0 = 0.5, sigma = 0.15), with sqrt(eps) noise added in the second case,
    leapfrog at dt = 5e-4 with BGT-1 at R = 1: finite after 1500 (1000 with noise) steps and
    below 20 (20 times the initial maximum with noise)."""
    N = 3
    a = wt.patch_mesh_arrays(wt.MESH_INFLATED_CUBE, N, 4, (0.1, 0.3, 1.0))
    o = oracle_from(O, N, a)
    x, y, z = o.coords()
    u, ud = O.ic_outgoing_pulse(x, y, z, 0.0, 1.0, 0.5, 0.15, 0.0, 0.0, 0.0)
    if noise:
        rng = np.random.default_rng(20260602)
        amp = np.sqrt(np.finfo(float).eps)
        u, ud = u + amp * rng.standard_normal(o.nn), ud + amp * rng.standard_normal(o.nn)
    bound = 20 * np.abs(u).max() if noise else 20.0
    dt = 5e-4
    ud = ud + 0.5 * dt * o.rhs_strong(u, ud, R=1.0)
    for _ in range(1000 if noise else 1500):
        u = u + dt * ud
        ud = ud + dt * o.rhs_strong(u, ud, R=1.0)
    assert np.all(np.isfinite(u)) and np.all(np.isfinite(ud))
    assert np.abs(u).max() < bound


def test_oracle_strong_form_cubed_cube_dirichlet(wt, O):
    """The reference's cubed-cube Dirichlet checks of the strong form
    (test/dirichlet_cubed_cube_tests.jl:54-109), on the oracle: the H_phys-weighted Rayleigh
    quotient of cos(pi x/2) cos(pi y/2) cos(pi z/2) on [-1, 1]^3 (N = 4, R = 0.3, zero
    Dirichlet faces) converges to 3 pi^2 / 4 with a geometric-mean ratio above 4 over
    M = 2, 4, 8, ending below 1e-3; at N = 3, M = 2 the spectrum has no growing mode
    (max Re < 1), is non-trivial (min Re < -1) and has bounded imaginary parts (< 100)."""
    lam = 3 * np.pi ** 2 / 4
    errs = []
    for M in (2, 4, 8):
        o = oracle_from(O, 4, wt.patch_mesh_arrays(wt.MESH_CUBED_CUBE, 4, M, (0.3,), outer_tag=1))
        x, y, z = o.coords()
        u = np.cos(np.pi * x / 2) * np.cos(np.pi * y / 2) * np.cos(np.pi * z / 2)
        H = o.get("Hphys")
        errs.append(abs(-np.dot(u, H * o.rhs_strong(u, np.zeros_like(u))) / np.dot(u, H * u) - lam))
    assert all(e > 0 for e in errs) and errs[-1] < errs[0]
    assert (errs[0] / errs[-1]) ** 0.5 > 4 and errs[-1] < 1e-3
    o = oracle_from(O, 3, wt.patch_mesh_arrays(wt.MESH_CUBED_CUBE, 3, 2, (0.3,), outer_tag=1))
    n = o.nn
    L = np.zeros((n, n))
    e, zero = np.zeros(n), np.zeros(n)
    for k in range(n):
        e[k] = 1.0
        L[:, k] = o.rhs_strong(e, zero)
        e[k] = 0.0
    ev = np.linalg.eigvals(L)
    assert ev.real.max() < 1.0 and ev.real.min() < -1.0 and np.abs(ev.imag).max() < 100.0


def test_oracle_strong_form_inflated_cube_dirichlet_j0(wt, O):
    """The reference's cubed-sphere Dirichlet checks of the strong form
    (test/dirichlet_cubed_sphere_tests.jl:84-128), on this library's inflated cube
    (L = 0.1, R1 = 0.3, R2 = 1, zero Dirichlet outer faces, N = 4): the H_phys-weighted
    Rayleigh quotient of j0(pi r) = sin(pi r) / (pi r) is within 1e-3 of pi^2 at M = 4, and
    its error shrinks more than 10 times from M = 2 to 4."""
    def rq(M):
        o = oracle_from(O, 4, wt.patch_mesh_arrays(wt.MESH_INFLATED_CUBE, 4, M, (0.1, 0.3, 1.0), outer_tag=1))
        x, y, z = o.coords()
        r = np.sqrt(x * x + y * y + z * z)
        u = np.where(r > 0, np.sin(np.pi * r) / np.where(r > 0, np.pi * r, 1.0), 1.0)
        H = o.get("Hphys")
        return -np.dot(u, H * o.rhs_strong(u, np.zeros_like(u))) / np.dot(u, H * u)

    errs = [abs(rq(M) - np.pi ** 2) for M in (2, 4)]
    assert all(e > 0 for e in errs)
    assert errs[1] / np.pi ** 2 < 1e-3 and errs[1] < errs[0] / 10
