"""Host logic of the z-slab partition (slabs.py), on the CPU: the layer ranges,
and the halo exchange -- every ghost layer receives the layer its neighbour owns
there, also on a periodic ring of two slabs, where each slab is the other's
upper and lower neighbour -- through a model of in-order point-to-point
delivery and through real gloo ranks (world sizes 2 and 3)."""
import os
import socket
import sys
from collections import defaultdict, deque

import pytest

from conftest import load_package

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("Mz,n,periodic", [(6, 1, False), (6, 2, False), (7, 3, False), (6, 2, True),
                                            (7, 3, True), (9, 4, True), (5, 5, False)])
def test_partition_covers_layers(Mz, n, periodic):
    S = load_package().slabs
    rs = S.partition(Mz, n, periodic)
    owned = [z for r in rs for z in range(r.own0, r.own0 + r.nown)]
    assert owned == list(range(Mz))
    assert max(r.nown for r in rs) - min(r.nown for r in rs) <= 1
    for r in rs:
        assert r.nz <= Mz
        if r.lower is not None:
            lo = rs[r.lower]
            assert (lo.own0 + lo.nown - 1) % Mz == r.z0 % Mz        # ghost below = neighbour's top layer
        else:
            assert r.own0 == 0 and not periodic or n == 1
        if r.upper is not None:
            up = rs[r.upper]
            assert up.own0 == (r.z0 + r.nz - 1) % Mz                 # ghost above = neighbour's bottom layer
    with pytest.raises(ValueError):
        S.partition(3, 4)


def test_partition_depth():
    S = load_package().slabs
    a, b = S.partition(14, 2, depth=6)
    assert (a.z0, a.nz, a.top_block, a.first_owned) == (0, 13, 1, 0)
    assert (b.z0, b.nz, b.top_block, b.first_owned) == (1, 13, 7, 6)
    rs = S.partition(18, 3, periodic=True, depth=6)
    assert [(r.z0, r.nz) for r in rs] == [(-6, 18), (0, 18), (6, 18)]
    with pytest.raises(ValueError):          # a slab must own the layers it lends
        S.partition(10, 2, depth=6)
    with pytest.raises(ValueError):          # no more layers than the mesh has
        S.partition(14, 2, periodic=True, depth=6)


def _field(r, Mz, width=4):
    # a slab's local layers: owned layers hold their whole-mesh layer number, ghosts -1
    return [[float(r.own0 + k - r.ghost_lo) if r.ghost_lo <= k < r.ghost_lo + r.nown else -1.0] * width
            for k in range(r.nz)]


@pytest.mark.parametrize("Mz,n,periodic,depth", [(6, 2, False, 1), (6, 2, True, 1), (7, 3, True, 1),
                                                  (8, 4, False, 1), (14, 2, False, 6), (18, 3, True, 6),
                                                  (9, 3, True, 2)])
def test_exchange_pairs_in_order(Mz, n, periodic, depth):
    """Every slab posts its messages (blocks of depth layers); delivery is in order per
    (sender, receiver) pair, as NCCL and gloo deliver point-to-point messages."""
    S = load_package().slabs
    rs = S.partition(Mz, n, periodic, depth)
    fields = [_field(r, Mz) for r in rs]
    wires = defaultdict(deque)
    for r in rs:   # phase 1: every slab posts its sends
        def send_recv(sends, recvs, r=r):
            for peer, buf in sends:
                wires[(r.index, peer)].append(list(buf))
        S.exchange(r, lambda layer, r=r: [row for row in fields[r.index][layer:layer + depth]],
                   lambda layer, buf: None, send_recv, list)
    for r in rs:   # phase 2: receives take messages in order
        def send_recv(sends, recvs, r=r):
            for peer, buf in recvs:
                buf.extend(wires[(peer, r.index)].popleft())
        def unpack(layer, buf, r=r):
            fields[r.index][layer:layer + depth] = buf
        S.exchange(r, lambda layer: None, unpack, send_recv, list)
    assert all(len(q) == 0 for q in wires.values())
    for r, f in zip(rs, fields):
        want = [float((r.z0 + k) % Mz) for k in range(r.nz)]
        assert [row[0] for row in f] == want


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, Mz, periodic, depth, q):
    import datetime
    import importlib.util
    import torch
    import torch.distributed as dist
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    from conftest import load_package as lp
    S = lp().slabs
    r = S.partition(Mz, world, periodic, depth)[rank]
    f = torch.tensor(_field(r, Mz, 5), dtype=torch.float64)
    for _ in range(3):   # repeated exchanges stay paired
        S.exchange(r, lambda layer: f[layer:layer + depth].flatten().clone(),
                   lambda layer, buf: f[layer:layer + depth].copy_(buf.view(depth, 5)),
                   S.dist_send_recv(dist), lambda: torch.empty(depth * 5, dtype=torch.float64))
    q.put((rank, f[:, 0].tolist(), [float((r.z0 + k) % Mz) for k in range(r.nz)]))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world,Mz,periodic,depth", [(2, 6, False, 1), (2, 6, True, 1), (3, 7, True, 1),
                                                      (3, 18, True, 6)])
def test_exchange_over_gloo(world, Mz, periodic, depth):
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, Mz, periodic, depth, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=180) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, got, want in out:
        assert got == want, rank


class _FaceSlab:
    """Stands in for slabs.Slab in DistFaceHalo: per local layer the two face planes
    (-z, +z) as one value each, owned layers holding 10 * global layer + face."""

    def __init__(self, r, Mz):
        import torch
        self.rng = r
        self.f = torch.full((r.nz, 2), -1.0, dtype=torch.float64)
        for z in range(r.first_owned, r.last_owned + 1):
            for k in range(2):
                self.f[z, k] = 10.0 * ((r.z0 + z) % Mz) + 4 + k
        self.bufs = {}

    def pack_face(self, st, layer, face):
        return self.f[layer, face - 4].reshape(1).clone()

    def unpack_face(self, st, layer, face, buf):
        self.f[layer, face - 4] = buf[0]

    def empty_face(self, which):
        import torch
        return self.bufs.setdefault(which, torch.empty(1, dtype=torch.float64))


def _face_worker(rank, world, port, Mz, periodic, q):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    from conftest import load_package as lp
    S = lp().slabs
    r = S.partition(Mz, world, periodic)[rank]
    s = _FaceSlab(r, Mz)
    halo = S.DistFaceHalo(s, dist)
    for st in range(3):   # repeated exchanges stay paired
        halo.start(st)
        halo.finish(st)
    lo = float(s.f[0, 1]) if r.lower is not None else None
    hi = float(s.f[r.nz - 1, 0]) if r.upper is not None else None
    want_lo = 10.0 * ((r.z0) % Mz) + 5 if r.lower is not None else None
    want_hi = 10.0 * ((r.z0 + r.nz - 1) % Mz) + 4 if r.upper is not None else None
    q.put((rank, (lo, hi), (want_lo, want_hi)))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world,Mz,periodic", [(2, 6, False), (3, 7, True), (2, 4, True)])
def test_face_halo_over_gloo(world, Mz, periodic):
    """DistFaceHalo: the +z face of every slab's top owned layer lands in the +z face of its
    upper neighbour's lower ghost layer, the -z face of its bottom owned layer in the -z face
    of its lower neighbour's upper ghost layer (the same elements), over gloo ranks."""
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_face_worker, args=(r, world, port, Mz, periodic, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=180) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, got, want in out:
        assert got == want, rank


@pytest.mark.parametrize("Mz,n,periodic", [(6, 2, False), (7, 3, True), (4, 3, False), (5, 1, False), (9, 4, True)])
def test_boundary_and_interior_layers_cover_owned(Mz, n, periodic):
    """The first stage half of step_faces runs on boundary_layers() then interior_runs(): together
    they cover every owned layer exactly once, the boundary ones are those next to a cut."""
    S = load_package().slabs

    for r in S.partition(Mz, n, periodic):
        s = object.__new__(S.Slab)  # the two methods need only .rng (no device objects)
        s.rng = r
        b = s.boundary_layers()
        runs = s.interior_runs()
        covered = list(b) + [z for z0, k in runs for z in range(z0, z0 + k)]
        assert sorted(covered) == list(range(r.first_owned, r.last_owned + 1))
        want = set()
        if r.lower is not None:
            want.add(r.first_owned)
        if r.upper is not None:
            want.add(r.last_owned)
        assert set(b) == want
        assert all(k > 0 for _, k in runs)
