"""Host logic of the z-slab decomposition: plane partition, slab layout (faces,
neighbours, ghost planes, body images) and the halo transport between processes,
run as gloo ranks on CPU with a stand-in domain whose messages name their sender."""
import socket

import numpy as np
import pytest
import torch

from lbm3d_bb_b200 import slab


def test_partition_is_balanced_and_complete():
    for nz in (3, 7, 30, 512):
        for parts in range(1, min(nz, 9) + 1):
            p = slab.partition(nz, parts)
            assert [z0 for z0, _ in p] == list(np.cumsum([0] + [n for _, n in p])[:-1])
            assert sum(n for _, n in p) == nz
            assert max(n for _, n in p) - min(n for _, n in p) <= 1
    with pytest.raises(ValueError):
        slab.partition(2, 3)


def test_layout_periodic_axis():
    lay = [slab.SlabLayout(30, 3, r) for r in range(3)]
    for r, L in enumerate(lay):
        assert L.faces_z == ("halo", "halo")
        assert L.nz_local == 12
        assert (L.lower, L.upper) == ((r - 1) % 3, (r + 1) % 3)
        z = L.global_planes()
        assert list(z[L.owned]) == list(range(10 * r, 10 * r + 10))
        assert z[0] == (10 * r - 1) % 30 and z[-1] == (10 * r + 10) % 30
        assert L.body_offsets() == [float(L.shift), L.shift - 30, L.shift + 30]
    two = [slab.SlabLayout(8, 2, r) for r in range(2)]
    assert (two[0].lower, two[0].upper, two[1].lower, two[1].upper) == (1, 1, 0, 0)


def test_layout_walled_axis():
    lay = [slab.SlabLayout(10, 3, r, ("wall", "pressure")) for r in range(3)]
    assert lay[0].faces_z == ("wall", "halo") and lay[0].lower is None and lay[0].upper == 1
    assert lay[1].faces_z == ("halo", "halo") and (lay[1].lower, lay[1].upper) == (0, 2)
    assert lay[2].faces_z == ("halo", "pressure") and lay[2].upper is None
    assert [L.nz_local for L in lay] == [5, 5, 4]
    assert list(lay[0].global_planes()) == [0, 1, 2, 3, 4]
    assert list(lay[2].global_planes()) == [6, 7, 8, 9]
    assert lay[1].body_offsets() == [float(lay[1].shift)]
    one = slab.SlabLayout(10, 1, 0, ("wall", "wall"))
    assert one.faces_z == ("wall", "wall") and one.nz_local == 10 and one.owned == slice(0, 10)
    with pytest.raises(ValueError):
        slab.SlabLayout(10, 2, 0, ("periodic", "wall"))


class _FakeDomain:
    """Messages are (sender rank, sender face, exchange number) as int64."""

    device = "cpu"
    halo_bytes = 24

    def __init__(self, rank):
        self.rank, self.count, self.got = rank, 0, {}

    def halo_pack(self, side, buf):
        buf.view(dtype=torch.int64)[:] = torch.tensor([self.rank, side, self.count])

    def halo_unpack(self, side, buf):
        self.got[(self.count, side)] = tuple(int(v) for v in buf.view(dtype=torch.int64))


def _rank(rank, world, port, z_faces, q):
    import torch.distributed as dist

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        lay = slab.SlabLayout(12, world, rank, z_faces)
        d = _FakeDomain(rank)
        ex = slab.SlabExchange(d, lay)
        for _ in range(3):
            ex.exchange()
            d.count += 1
        q.put((rank, d.got))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,z_faces", [(2, ("periodic", "periodic")), (3, ("periodic", "periodic")),
                                           (3, ("wall", "wall"))])
def test_exchange_delivers_each_face_its_neighbours_message(world, z_faces):
    import multiprocessing as mp

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, z_faces, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in range(world):
        lay = slab.SlabLayout(12, world, r, z_faces)
        want = {}
        for k in range(3):
            if lay.lower is not None:
                want[(k, 0)] = (lay.lower, 1, k)  # the z-lo ghost takes the lower slab's z-hi message
            if lay.upper is not None:
                want[(k, 1)] = (lay.upper, 0, k)
        assert got[r] == want, (r, got[r])
