"""z-slab decomposition of one box over several GPUs (one process per GPU).

Replaces the reference's multi-GPU path: METIS partitioning (Partitioning.jl:107-119)
and the MPI halo exchange called from the time loop (begin_halo_exchange! /
finish_halo_exchange!, Exchange.jl:11-107, called at MainCore.jl:272-286).

Slab r owns the global planes z0 .. z0 + n - 1 and keeps one ghost plane on every z face
that borders another slab (face kind "halo").  After every step each slab packs one
message per halo face (`Domain.halo_pack`), the message crosses to the neighbouring
slab, and the neighbour merges it (`Domain.halo_unpack`): one exchange per step of
5 populations x nx x ny per face, in the storage type.  The kernels of a slab are the
single-domain kernels; ghost planes are read and written by their neighbours but never
updated, so a decomposed run reproduces the undivided run node for node.

Bodies are static and given in global coordinates.  On a globally periodic z axis each
body is also placed at z - nz and z + nz (the undivided box measures distances to the
nearest image along a periodic axis), so bodies that cross the wrap appear in both slabs.

Transports: `SlabGroup` holds several slabs of one process (one GPU, or several GPUs
driven from one process) and hands the messages over directly; `SlabExchange` moves
them between processes with torch.distributed point-to-point operations (NCCL between
GPUs over NVLink; gloo between CPU processes for the host-logic tests).
"""
from __future__ import annotations

from typing import Optional, Sequence

import numpy as np

from . import abi


def partition(nz: int, parts: int) -> list[tuple[int, int]]:
    """(first plane, plane count) of each slab: counts differ by at most one."""
    if parts < 1 or nz < parts:
        raise ValueError(f"cannot split {nz} planes into {parts} slabs")
    base, extra = divmod(nz, parts)
    out, z0 = [], 0
    for r in range(parts):
        n = base + (1 if r < extra else 0)
        out.append((z0, n))
        z0 += n
    return out


class SlabLayout:
    """Host-side geometry of slab `rank` of `parts` along a z axis of `nz` planes whose
    global faces are `z_faces` (two face names)."""

    def __init__(self, nz: int, parts: int, rank: int, z_faces: Sequence[str] = ("periodic", "periodic")):
        if not 0 <= rank < parts:
            raise ValueError("rank out of range")
        if (z_faces[0] == "periodic") != (z_faces[1] == "periodic"):
            raise ValueError("both z faces periodic or neither")
        self.nz, self.parts, self.rank = nz, parts, rank
        self.periodic = z_faces[0] == "periodic"
        self.z0, self.n = partition(nz, parts)[rank]
        if parts == 1:
            self.lo_halo = self.hi_halo = False
        else:
            self.lo_halo = self.periodic or rank > 0
            self.hi_halo = self.periodic or rank < parts - 1
        self.faces_z = ("halo" if self.lo_halo else z_faces[0], "halo" if self.hi_halo else z_faces[1])
        self.nz_local = self.n + int(self.lo_halo) + int(self.hi_halo)
        self.lower: Optional[int] = (rank - 1) % parts if self.lo_halo else None
        self.upper: Optional[int] = (rank + 1) % parts if self.hi_halo else None
        self.shift = int(self.lo_halo) - self.z0  # local z = global z + shift

    @property
    def owned(self) -> slice:
        """Local planes this slab owns."""
        return slice(int(self.lo_halo), int(self.lo_halo) + self.n)

    def global_planes(self) -> np.ndarray:
        """Global z of every local plane (ghost planes included, wrapped on a periodic axis)."""
        z = np.arange(self.nz_local) - self.shift
        return z % self.nz if self.periodic else z

    def body_offsets(self) -> list[float]:
        """z shifts that place a global body in this slab, the body itself first (the
        first body placed is the torque centre), then its periodic images."""
        if self.periodic and self.parts > 1:
            return [float(self.shift), self.shift - self.nz, self.shift + self.nz]
        return [float(self.shift)]


class SlabDomain:
    """One slab: a `Domain` of nx x ny x nz_local nodes with halo z faces.

    Keyword arguments other than `faces` go to `Domain` unchanged."""

    def __init__(self, nx: int, ny: int, nz: int, parts: int, rank: int, *, faces=("periodic",) * 6, **kw):
        from .domain import Domain

        faces = tuple(faces)
        self.layout = SlabLayout(nz, parts, rank, faces[4:6])
        self.shape_global = (nx, ny, nz)
        self.domain = Domain(nx, ny, self.layout.nz_local, faces=faces[:4] + self.layout.faces_z, **kw)

    def close(self) -> None:
        self.domain.close()

    # -- geometry (global coordinates) ------------------------------------------------------
    def add_body(self, body: abi.LbmBody) -> None:
        if body.moving:
            raise ValueError("slabs take static bodies only")
        for dz in self.layout.body_offsets():
            b = abi.LbmBody.from_buffer_copy(body)
            b.center[2] = body.center[2] + dz
            self.domain.add_body(b)

    def add_spheres(self, xyzr: np.ndarray) -> None:
        a = np.asarray(xyzr, dtype=np.float64).reshape(-1, 4)
        parts = []
        for dz in self.layout.body_offsets():
            s = a.copy()
            s[:, 2] += dz
            parts.append(s)
        self.domain.add_spheres(np.concatenate(parts))

    # -- state ------------------------------------------------------------------------------
    def init_equilibrium(self, rho=None, u=None, v=None, w=None) -> None:
        """Equilibrium at the given fields: scalars or global (nz, ny, nx) arrays."""
        zs = self.layout.global_planes()

        def local(a):
            if a is None or np.ndim(a) == 0:
                return a
            return np.ascontiguousarray(np.asarray(a)[zs]).ravel()

        self.domain.init_equilibrium(local(rho), local(u), local(v), local(w))

    def macros(self):
        """(rho, u, v, w) of the owned planes, shape (n, ny, nx) each."""
        return tuple(m[self.layout.owned] for m in self.domain.macros())

    def populations(self):
        """(19, n, ny, nx) populations of the owned planes (FP64, canonical)."""
        f = self.domain.populations().reshape(19, self.layout.nz_local, self.shape_global[1], self.shape_global[0])
        return f[:, self.layout.owned]

    def force(self, step: Optional[int] = None) -> np.ndarray:
        """This slab's part of the body force / torque (sum the slabs for the total)."""
        return self.domain.force(step)

    # -- halo messages ----------------------------------------------------------------------
    def sides(self) -> list[int]:
        return [s for s, h in ((0, self.layout.lo_halo), (1, self.layout.hi_halo)) if h]

    def neighbour(self, side: int) -> int:
        return self.layout.lower if side == 0 else self.layout.upper


class SlabGroup:
    """Every slab of a box in one process; messages pass directly from the packing
    slab's buffer to the neighbour's unpack, in stream order (one stream for all)."""

    def __init__(self, slabs: Sequence[SlabDomain]):
        import torch

        self.slabs = list(slabs)
        if [s.layout.rank for s in self.slabs] != list(range(len(self.slabs))):
            raise ValueError("slabs must be given in rank order")
        dev = self.slabs[0].domain.device
        self.buf = {(r, side): torch.empty(s.domain.halo_bytes, dtype=torch.uint8, device=f"cuda:{dev}")
                    for r, s in enumerate(self.slabs) for side in s.sides()}

    def exchange(self) -> None:
        for r, s in enumerate(self.slabs):
            for side in s.sides():
                s.domain.halo_pack(side, self.buf[(r, side)])
        for r, s in enumerate(self.slabs):
            for side in s.sides():
                s.domain.halo_unpack(side, self.buf[(s.neighbour(side), 1 - side)])

    def step(self, n: int = 1) -> None:
        for _ in range(n):
            for s in self.slabs:
                s.domain.step(1)
            self.exchange()

    def force(self, step: Optional[int] = None) -> np.ndarray:
        return sum(s.force(step) for s in self.slabs)


class SlabExchange:
    """Halo transport of one slab per process over torch.distributed.

    `domain` needs halo_bytes, halo_pack(side, buf), halo_unpack(side, buf) and a
    `device` ("cpu" or a CUDA index); `layout` is the slab's SlabLayout.  Every rank
    issues its sends (z-hi face first) and then its receives (z-lo face first), so when
    both neighbours are the same rank (two slabs on a periodic axis) the first message
    between the pair is the one for the receiver's z-lo face.  NCCL has no message tags:
    this order is what pairs them."""

    def __init__(self, domain, layout: SlabLayout, group=None):
        import torch

        self.d, self.layout, self.group = domain, layout, group
        dev = domain.device
        device = "cpu" if dev == "cpu" else f"cuda:{dev}"
        nb = int(domain.halo_bytes)
        self.sides = [s for s, h in ((0, layout.lo_halo), (1, layout.hi_halo)) if h]
        self.send = {s: torch.empty(nb, dtype=torch.uint8, device=device) for s in self.sides}
        self.recv = {s: torch.empty(nb, dtype=torch.uint8, device=device) for s in self.sides}

    def _peer(self, side: int) -> int:
        import torch.distributed as dist

        r = self.layout.lower if side == 0 else self.layout.upper
        return r if self.group is None else dist.get_global_rank(self.group, r)

    def exchange(self) -> None:
        import torch.distributed as dist

        if not self.sides:
            return
        for s in self.sides:
            self.d.halo_pack(s, self.send[s])
        # torch.distributed orders its transfers after the caller's current stream; the
        # packs ran on the domain's stream, which may be another one: hand over with events
        # (domain stream -> current stream before the sends, back before the unpacks)
        dstream = self._domain_stream()
        if dstream is not None:
            import torch

            packed = torch.cuda.Event()
            packed.record(dstream)
            torch.cuda.current_stream(dstream.device).wait_event(packed)
        ops = [dist.P2POp(dist.isend, self.send[s], self._peer(s), self.group) for s in sorted(self.sides, reverse=True)]
        ops += [dist.P2POp(dist.irecv, self.recv[s], self._peer(s), self.group) for s in sorted(self.sides)]
        for req in dist.batch_isend_irecv(ops):
            req.wait()
        if dstream is not None:
            received = torch.cuda.Event()
            received.record(torch.cuda.current_stream(dstream.device))
            dstream.wait_event(received)
        for s in self.sides:
            self.d.halo_unpack(s, self.recv[s])

    def _domain_stream(self):
        """The torch stream the domain enqueues on (its own, or the legacy default stream
        when it has none); None for a CPU domain."""
        if self.d.device == "cpu":
            return None
        import torch

        s = getattr(self.d, "stream", None)
        return s if s is not None else torch.cuda.default_stream(int(self.d.device))


def run(argv=None) -> None:
    """Porous periodic box decomposed into z-slabs, one per process (torchrun):
    prints the whole-box MLUPS (device time, max over ranks) and the total drag."""
    import argparse
    import os

    import torch
    import torch.distributed as dist

    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=256, help="box edge (nodes)")
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=4)
    ap.add_argument("--storage", default="fp32", choices=["fp32", "fp64", "fp16dev"])
    ap.add_argument("--spheres", type=int, default=25)
    args = ap.parse_args(argv)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    n = args.n
    rng = np.random.default_rng(3)
    xyzr = np.column_stack([rng.uniform(0, n, (args.spheres, 3)), rng.uniform(6, 16, args.spheres)])
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        s = SlabDomain(n, n, n, world, rank, collision="BGK", storage=args.storage, omega_p=1.0 / 0.6,
                       accel=(1e-6, 0.0, 0.0), compute_force=True, device=local, stream=stream)
        s.add_spheres(xyzr)
        s.init_equilibrium()
        ex = SlabExchange(s.domain, s.layout)
        for _ in range(args.warmup):
            s.domain.step(1)
            ex.exchange()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(args.steps):
            s.domain.step(1)
            ex.exchange()
        e1.record(stream)
        torch.cuda.synchronize()
        ms = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64, device=f"cuda:{local}")
        fz = torch.tensor(s.force(), dtype=torch.float64, device=f"cuda:{local}")
        if world > 1:
            dist.all_reduce(ms, op=dist.ReduceOp.MAX)
            dist.all_reduce(fz)
        if rank == 0:
            mlups = n ** 3 * args.steps / (ms.item() * 1e-3) / 1e6
            print(f"slabs={world} box={n}^3 {args.storage}: {mlups:.0f} MLUPS, drag {fz[0].item():.6e}", flush=True)
        s.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    run()
