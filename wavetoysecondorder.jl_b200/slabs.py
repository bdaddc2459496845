"""One solve of the analytic (warped) cube split into z-slabs of element layers.

No counterpart in the reference, whose evolve3d (src/evolve.jl:1149-1358) runs a
solve on one device.  Slab s owns a run of consecutive element layers and holds
one ghost layer beyond each cut (the layer its neighbour slab owns there).  An
RK4 stage is split in two halves (wt_rk4_stage_curved): after the first
(gradient, flux, Phi stage update) every slab sends the layers next to its cuts
-- the Phi the next stage reads and the three flux components, one packed
buffer per layer (wt_halo_copy) -- to its neighbours, which unpack them into
their ghost layers; the second half (divergence, Pi stage update) then reads
correct neighbour traces, and so does the next stage's first half.  That is
one halo exchange per RK4 stage.  The owned layers of every slab advance
exactly as in the undivided mesh; ghost layers hold scratch values otherwise.

With Kreiss-Oliger dissipation (eps_KO != 0) the z passes of D^6 reach six
element layers, so the partition keeps depth = 6 ghost layers beyond each cut.
Every stage then runs whole on each slab (wt_rk4_stage_curved_ko), after which
the state the next stage reads is exchanged, six layers per cut (step_ko).  The
slabs take the whole mesh's mu (Workspace.set_mu).

Slabs live either all in one process on one device (LocalHalo: the exchange is
a device copy per cut) or one per rank (DistHalo: torch.distributed point-to-
point messages, NCCL between GPUs).
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Callable, List, Optional, Sequence

from . import wavetoy as wt


@dataclass(frozen=True)
class SlabRange:
    """Layers of slab `index` in the whole mesh's numbering: it owns own0 .. own0 + nown - 1
    and holds z0 .. z0 + nz - 1 (z0 may be negative for a periodic mesh: taken modulo Mz)."""
    index: int
    own0: int
    nown: int
    lower: Optional[int]   # slab owning the layers below (None: outer face or no neighbour)
    upper: Optional[int]
    depth: int = 1         # ghost layers beyond each cut

    @property
    def ghost_lo(self) -> int:
        return 0 if self.lower is None else self.depth

    @property
    def ghost_hi(self) -> int:
        return 0 if self.upper is None else self.depth

    @property
    def z0(self) -> int:
        return self.own0 - self.ghost_lo

    @property
    def nz(self) -> int:
        return self.nown + self.ghost_lo + self.ghost_hi

    # local layer numbers (0 .. nz - 1)
    @property
    def first_owned(self) -> int:
        return self.ghost_lo

    @property
    def last_owned(self) -> int:
        return self.ghost_lo + self.nown - 1

    @property
    def top_block(self) -> int:
        """First local layer of the depth owned layers its upper neighbour holds as ghosts."""
        return self.ghost_lo + self.nown - self.depth


def partition(Mz: int, nslabs: int, periodic: bool = False, depth: int = 1) -> List[SlabRange]:
    """Split Mz element layers into nslabs runs as equal as possible (the first Mz mod
    nslabs slabs get one more); periodic meshes close the ring of slabs.  depth ghost
    layers beyond each cut (1 for the RHS alone, 6 with Kreiss-Oliger dissipation)
    must come from the neighbour's own layers, so every slab owns at least depth."""
    if nslabs < 1 or nslabs > Mz:
        raise ValueError("need 1 <= nslabs <= Mz")
    if depth < 1:
        raise ValueError("depth must be >= 1")
    base, rem = divmod(Mz, nslabs)
    out, z = [], 0
    for r in range(nslabs):
        n = base + (1 if r < rem else 0)
        lower = r - 1 if r > 0 else (nslabs - 1 if periodic and nslabs > 1 else None)
        upper = r + 1 if r < nslabs - 1 else (0 if periodic and nslabs > 1 else None)
        rng = SlabRange(r, z, n, lower, upper, depth)
        if rng.nz > Mz:
            raise ValueError(f"slab {r} would hold {rng.nz} layers of {Mz}: use fewer slabs")
        if nslabs > 1 and n < depth:
            raise ValueError(f"slab {r} owns {n} layers, fewer than the {depth} ghost layers it supplies")
        out.append(rng)
        z += n
    return out


def exchange(rng: SlabRange, pack: Callable[[int], object], unpack: Callable[[int, object], None],
             send_recv: Callable[[list, list], None], empty: Callable[[], object]):
    """One halo exchange of slab rng with its neighbours.  pack(layer) gives the packed
    buffer of the rng.depth local layers from `layer`, unpack(layer, buf) writes one
    back, empty() a receive buffer;
    send_recv(sends, recvs) moves [(slab, buffer)] pairs.  Messages are posted in two
    phases -- every slab sends its top owned layer up while receiving its bottom ghost
    from below, then its bottom owned layer down while receiving its top ghost from
    above -- so that between any two slabs (two slabs of a periodic ring are each
    other's upper and lower neighbour) sends and receives pair up in order."""
    sends, recvs = [], []
    if rng.upper is not None:
        sends.append((rng.upper, pack(rng.top_block)))
    if rng.lower is not None:
        recvs.append((rng.lower, 0, empty()))
    if rng.lower is not None:
        sends.append((rng.lower, pack(rng.first_owned)))
    if rng.upper is not None:
        recvs.append((rng.upper, rng.nz - rng.depth, empty()))
    send_recv(sends, [(peer, buf) for peer, _, buf in recvs])
    for _, layer, buf in recvs:
        unpack(layer, buf)


def dist_send_recv(dist, group=None, rank_of: Callable[[int], int] = lambda s: s):
    """send_recv for exchange() over torch.distributed: every send and receive as one
    batch of point-to-point operations (NCCL runs a batch as one group), sends to a
    peer in the order exchange() lists them and receives from a peer likewise."""
    def go(sends, recvs):
        ops = []
        # interleave per exchange() phase: (send up, recv from below), (send down, recv from above)
        order = []
        for k in range(max(len(sends), len(recvs))):
            if k < len(sends):
                order.append(("s", sends[k]))
            if k < len(recvs):
                order.append(("r", recvs[k]))
        for kind, (peer, buf) in order:
            op = dist.isend if kind == "s" else dist.irecv
            ops.append(dist.P2POp(op, buf, rank_of(peer), group))
        if ops:
            for w in dist.batch_isend_irecv(ops):
                w.wait()
    return go


class Slab:
    """One slab's device objects: mesh (wt_mesh_create_slab), static background,
    workspace and state; ghost layers included."""

    def __init__(self, ctx, rng: SlabRange, N: int, M, x0: float = 0.0, x1: float = 1.0, *, warp_A: float = 0.0,
                 periodic: bool = False, outer_tag: int = 0, precision: int = wt.WT_F64,
                 bg_kind: int = wt.BG_MINKOWSKI, bg_params: Sequence[float] = (), fp32_form: Optional[int] = None,
                 mu: Optional[float] = None):
        M = (M, M, M) if isinstance(M, int) else tuple(M)
        self.rng = rng
        self.ctx = ctx
        self.mesh = wt.Mesh.slab(ctx, N, M, rng.z0, rng.nz, x0, x1, periodic=periodic, outer_tag=outer_tag,
                                 warp_A=warp_A, precision=precision)
        if precision == wt.WT_F32 and fp32_form is not None:
            self.mesh.set_fp32_form(fp32_form)
        self.coef = wt.sample_background3d(self.mesh, bg_kind, bg_params)
        self.ws = wt.make_wave3d_workspace(self.mesh)
        if mu is not None:
            self.ws.set_mu(mu)
        self.Phi, self.Pi = self.mesh.zeros(), self.mesh.zeros()
        self.layer_nodes = M[0] * M[1] * N ** 3
        # halo buffers, allocated on first use and reused by every exchange: one
        # send buffer per packed layer, two receive buffers used in turn
        # (an exchange posts at most two receives and completes them before it returns)
        self._send = {}
        self._recv = {}
        self._recv_turn = {}

    def owned(self, field):
        """The owned layers of a local field (a view)."""
        a = self.rng.first_owned * self.layer_nodes
        return field[a:a + self.rng.nown * self.layer_nodes]

    def stage(self, dt: float, st: int, part: int, bc3d=None, metric: bool = True):
        wt.rk4_stage_curved(self.Phi, self.Pi, self.coef, self.ws, dt, st, part, bc3d=bc3d, metric=metric)

    def _new(self, kind: str):
        import torch
        n = wt.halo_size(self.ws) if kind == "flux" else 2 * self.rng.depth * self.layer_nodes
        return torch.empty(n, dtype=self.mesh.dtype, device=self.Phi.device)

    def _send_buf(self, kind: str, layer: int):
        key = (kind, layer)
        if key not in self._send:
            self._send[key] = self._new(kind)
        return self._send[key]

    def _recv_buf(self, kind: str):
        if kind not in self._recv:
            self._recv[kind] = (self._new(kind), self._new(kind))
            self._recv_turn[kind] = 0
        t = self._recv_turn[kind]
        self._recv_turn[kind] = t ^ 1
        return self._recv[kind][t]

    def empty(self):
        """A receive buffer of the flux halo (one of two reused in turn)."""
        return self._recv_buf("flux")

    def pack(self, st: int, layer: int):
        buf = self._send_buf("flux", layer)
        wt.halo_copy(self.ws, self.Phi, st, layer, buf, True)
        return buf

    def unpack(self, st: int, layer: int, buf):
        wt.halo_copy(self.ws, self.Phi, st, layer, buf, False)

    # the face-plane halo (step_faces): both stage halves run on the owned layers only
    def stage_layers(self, dt: float, st: int, part: int, layer0: int, nlayers: int, bc3d=None,
                     metric: bool = True):
        if nlayers > 0:
            wt.rk4_stage_curved_layers(self.Phi, self.Pi, self.coef, self.ws, dt, st, part, layer0, nlayers,
                                       bc3d=bc3d, metric=metric)

    def boundary_layers(self):
        """The owned layers next to a cut (their face planes are sent)."""
        r = self.rng
        out = []
        if r.lower is not None:
            out.append(r.first_owned)
        if r.upper is not None and r.last_owned not in out:
            out.append(r.last_owned)
        return out

    def interior_runs(self):
        """(layer0, nlayers) runs of the owned layers not next to a cut."""
        b = set(self.boundary_layers())
        runs, start = [], None
        for z in range(self.rng.first_owned, self.rng.last_owned + 2):
            inside = z <= self.rng.last_owned and z not in b
            if inside and start is None:
                start = z
            elif not inside and start is not None:
                runs.append((start, z - start))
                start = None
        return runs

    def _face_buf(self, key):
        import torch
        if key not in self._send:
            self._send[key] = torch.empty(wt.halo_face_size(self.ws), dtype=self.mesh.dtype, device=self.Phi.device)
        return self._send[key]

    def pack_face(self, st: int, layer: int, face: int):
        buf = self._face_buf(("face", layer, face))
        wt.halo_face_copy(self.ws, self.Phi, st, layer, face, buf, True)
        return buf

    def unpack_face(self, st: int, layer: int, face: int, buf):
        wt.halo_face_copy(self.ws, self.Phi, st, layer, face, buf, False)

    def empty_face(self, which: str):
        """The receive buffer of the face halo from below ("lo") or above ("hi")."""
        return self._face_buf(("recv", which))

    # the state halo of the dissipative stepping (depth layers of Phi and Pi)
    def stage_ko(self, dt: float, st: int, eps_KO: float, bc3d=None, metric: bool = True):
        wt.rk4_stage_curved_ko(self.Phi, self.Pi, self.coef, self.ws, dt, st, eps_KO, bc3d=bc3d, metric=metric)

    def empty_state(self):
        """A receive buffer of the state halo (one of two reused in turn)."""
        return self._recv_buf("state")

    def pack_state(self, st: int, layer: int):
        buf = self._send_buf("state", layer)
        wt.halo_state_copy(self.ws, self.Phi, self.Pi, st, layer, self.rng.depth, buf, True)
        return buf

    def unpack_state(self, st: int, layer: int, buf):
        wt.halo_state_copy(self.ws, self.Phi, self.Pi, st, layer, self.rng.depth, buf, False)

    def close(self):
        for o in (self.ws, self.coef, self.mesh):
            o.close()


class LocalHalo:
    """All slabs in this process, on one device: each message is a device copy."""

    def __init__(self, slabs: List[Slab]):
        self.slabs = slabs

    def __call__(self, st: int):
        msgs = {}
        for s in self.slabs:   # the layers next to each cut, packed ...
            r = s.rng
            if r.upper is not None:
                msgs[(r.index, "up")] = s.pack(st, r.last_owned)
            if r.lower is not None:
                msgs[(r.index, "down")] = s.pack(st, r.first_owned)
        for s in self.slabs:   # ... into the neighbours' ghost layers
            r = s.rng
            if r.lower is not None:
                s.unpack(st, 0, msgs[(r.lower, "up")])
            if r.upper is not None:
                s.unpack(st, r.nz - 1, msgs[(r.upper, "down")])


class DistHalo:
    """One slab per rank (rank = slab index): torch.distributed point-to-point."""

    def __init__(self, slab: Slab, dist, group=None):
        self.slab, self.dist, self.group = slab, dist, group

    def __call__(self, st: int):
        s = self.slab
        exchange(s.rng, lambda layer: s.pack(st, layer), lambda layer, buf: s.unpack(st, layer, buf),
                 dist_send_recv(self.dist, self.group), s.empty)


class LocalStateHalo:
    """The state halo (depth layers of Phi and Pi) between slabs of this process."""

    def __init__(self, slabs: List[Slab]):
        self.slabs = slabs

    def __call__(self, st: int):
        msgs = {}
        for s in self.slabs:
            r = s.rng
            if r.upper is not None:
                msgs[(r.index, "up")] = s.pack_state(st, r.top_block)
            if r.lower is not None:
                msgs[(r.index, "down")] = s.pack_state(st, r.first_owned)
        for s in self.slabs:
            r = s.rng
            if r.lower is not None:
                s.unpack_state(st, 0, msgs[(r.lower, "up")])
            if r.upper is not None:
                s.unpack_state(st, r.nz - r.depth, msgs[(r.upper, "down")])


class DistStateHalo:
    """The state halo, one slab per rank, over torch.distributed."""

    def __init__(self, slab: Slab, dist, group=None):
        self.slab, self.dist, self.group = slab, dist, group

    def __call__(self, st: int):
        s = self.slab
        exchange(s.rng, lambda layer: s.pack_state(st, layer), lambda layer, buf: s.unpack_state(st, layer, buf),
                 dist_send_recv(self.dist, self.group), s.empty_state)


def exchange_faces(rng: SlabRange, pack_up: Callable[[], object], pack_down: Callable[[], object],
                   recv_lo: object, recv_hi: object, send_recv: Callable[[list, list], None]):
    """Post the face-plane messages of slab rng in exchange()'s two-phase order: the +z face
    of its top owned layer up while receiving its lower ghost's face from below, then the
    -z face of its bottom owned layer down while receiving its upper ghost's face from above."""
    sends, recvs = [], []
    if rng.upper is not None:
        sends.append((rng.upper, pack_up()))
    if rng.lower is not None:
        recvs.append((rng.lower, recv_lo))
    if rng.lower is not None:
        sends.append((rng.lower, pack_down()))
    if rng.upper is not None:
        recvs.append((rng.upper, recv_hi))
    return send_recv(sends, recvs)


class LocalFaceHalo:
    """The face-plane halo between slabs of this process (device copies).  start()
    packs every slab's boundary faces and unpacks them into the neighbours' ghost
    faces; finish() has nothing left to do."""

    def __init__(self, slabs: List[Slab]):
        self.slabs = slabs

    def start(self, st: int):
        msgs = {}
        for s in self.slabs:
            r = s.rng
            if r.upper is not None:
                msgs[(r.index, "up")] = s.pack_face(st, r.last_owned, 5)
            if r.lower is not None:
                msgs[(r.index, "down")] = s.pack_face(st, r.first_owned, 4)
        for s in self.slabs:
            r = s.rng
            if r.lower is not None:
                s.unpack_face(st, 0, 5, msgs[(r.lower, "up")])
            if r.upper is not None:
                s.unpack_face(st, r.nz - 1, 4, msgs[(r.upper, "down")])

    def finish(self, st: int):
        pass


class DistFaceHalo:
    """The face-plane halo, one slab per rank, over torch.distributed.  start() packs and
    posts the messages as one batch of point-to-point operations (NCCL runs them on its
    own stream, after the packs); finish() makes the current stream wait for them and
    unpacks -- so that work enqueued in between (the interior layers' first stage half)
    overlaps the transfer."""

    def __init__(self, slab: Slab, dist, group=None, rank_of: Callable[[int], int] = lambda s: s):
        self.slab, self.dist, self.group, self.rank_of = slab, dist, group, rank_of
        self._works = []

    def start(self, st: int):
        s, r = self.slab, self.slab.rng

        def post(sends, recvs):
            order = []
            for k in range(max(len(sends), len(recvs))):
                if k < len(sends):
                    order.append((self.dist.isend, sends[k]))
                if k < len(recvs):
                    order.append((self.dist.irecv, recvs[k]))
            ops = [self.dist.P2POp(op, buf, self.rank_of(peer), self.group) for op, (peer, buf) in order]
            self._works = self.dist.batch_isend_irecv(ops) if ops else []

        self._lo = s.empty_face("lo") if r.lower is not None else None
        self._hi = s.empty_face("hi") if r.upper is not None else None
        exchange_faces(r, lambda: s.pack_face(st, r.last_owned, 5), lambda: s.pack_face(st, r.first_owned, 4),
                       self._lo, self._hi, post)

    def finish(self, st: int):
        for w in self._works:
            w.wait()
        self._works = []
        s, r = self.slab, self.slab.rng
        if r.lower is not None:
            s.unpack_face(st, 0, 5, self._lo)
        if r.upper is not None:
            s.unpack_face(st, r.nz - 1, 4, self._hi)


def step_faces(slabs: List[Slab], halo, dt: float, nsteps: int, bc3d=None, metric: bool = True):
    """nsteps RK4 steps of the partitioned solve with the face-plane halo (depth-1
    partitions, eps_KO = 0): per stage the first half on the owned layers next to a cut,
    the exchange started, the first half on the other owned layers (overlapping the
    transfer when the halo is asynchronous), the exchange finished, the second half on
    the owned layers.  Ghost layers are never computed: only the face planes the owned
    elements read are written into them.  The ghost layers of the starting state must
    hold the state (as after set-up from the analytic initial data on the whole slab)."""
    if any(s.rng.depth != 1 for s in slabs):
        raise ValueError("the face halo serves depth-1 partitions")
    for _ in range(int(nsteps)):
        for st in range(4):
            for s in slabs:
                for z in s.boundary_layers():
                    s.stage_layers(dt, st, 1, z, 1, bc3d, metric)
            halo.start(st)
            for s in slabs:
                for z0, nz in s.interior_runs():
                    s.stage_layers(dt, st, 1, z0, nz, bc3d, metric)
            halo.finish(st)
            for s in slabs:
                s.stage_layers(dt, st, 2, s.rng.first_owned, s.rng.nown, bc3d, metric)


def step_ko(slabs: List[Slab], halo, dt: float, nsteps: int, eps_KO: float, bc3d=None, metric: bool = True):
    """nsteps RK4 steps with Kreiss-Oliger dissipation: every stage whole on each slab,
    then the state halo (depth 6).  The ghost layers of the starting state are
    exchanged first, so any state the owners hold can start it."""
    if any(s.rng.depth < 6 for s in slabs if s.rng.lower is not None or s.rng.upper is not None):
        raise ValueError("dissipation on slabs needs partition(..., depth=6)")
    halo(3)
    for _ in range(int(nsteps)):
        for st in range(4):
            for s in slabs:
                s.stage_ko(dt, st, eps_KO, bc3d, metric)
            halo(st)


def step(slabs: List[Slab], halo, dt: float, nsteps: int, bc3d=None, metric: bool = True):
    """nsteps RK4 steps of the partitioned solve (the slabs this process holds; depth-1
    partitions, eps_KO = 0)."""
    if any(s.rng.depth != 1 for s in slabs):
        raise ValueError("the flux halo is one layer deep: use step_ko for a depth-6 partition")
    for _ in range(int(nsteps)):
        for st in range(4):
            for s in slabs:
                s.stage(dt, st, 1, bc3d, metric)
            halo(st)
            for s in slabs:
                s.stage(dt, st, 2, bc3d, metric)
