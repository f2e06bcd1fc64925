"""z-slab decomposition on one GPU: the box split into 2 and 3 slabs (ghost planes on
halo faces, one halo exchange per step, messages handed over in stream order) against
the undivided box — the populations of every owned node and the summed body force,
after odd and even step counts, on periodic and walled z axes — and the C ABI's error
paths for halo faces."""
import numpy as np
import pytest

from lbm3d_bb_b200 import Domain, abi
from lbm3d_bb_b200._capi import LbmError
from lbm3d_bb_b200.slab import SlabDomain, SlabGroup
from tests import cases
from tests.cases import rel_l2

pytestmark = pytest.mark.gpu

NX, NY, NZ = 24, 20, 30
# spheres crossing the slab boundaries of 2 and 3 slabs (z = 10, 15, 20) and the periodic
# wrap (z = 0), one inside a slab
SPHERES = np.array([[6.3, 7.1, 10.2, 4.2], [15.5, 12.4, 15.1, 3.6], [9.2, 4.8, 19.7, 3.9], [18.1, 15.2, 0.6, 4.4],
                    [12.0, 10.0, 5.0, 2.5]])
TOL = {"fp64": 1e-13, "fp32": 1e-6, "fp16dev": 1e-4}
CHANNEL = ("inlet", "pressure", "wall", "wall", "wall", "wall")


def _kw(storage, collision, faces):
    kw = dict(collision=collision, storage=storage, faces=faces, omega_p=1.0 / 0.6, compute_force=True)
    if collision == "TRT":
        kw["omega_m"] = 1.0 / (0.5 + 0.1875 / (0.6 - 0.5))
    if faces == CHANNEL:
        kw["face_u"] = [(0.05, 0.0, 0.0)] + [(0.0, 0.0, 0.0)] * 5
    else:
        kw["accel"] = (1e-5, 0.0, 0.0)
    return kw


def _full(steps, storage, collision, faces):
    d = Domain(NX, NY, NZ, **_kw(storage, collision, faces))
    d.add_spheres(SPHERES)
    d.init_equilibrium()
    d.step(steps)
    return d


def _slabs(parts, steps, storage, collision, faces):
    slabs = [SlabDomain(NX, NY, NZ, parts, r, **_kw(storage, collision, faces)) for r in range(parts)]
    for s in slabs:
        s.add_spheres(SPHERES)
        s.init_equilibrium()
    g = SlabGroup(slabs)
    g.step(steps)
    return g


@pytest.mark.parametrize("parts,steps,storage,collision,faces", [
    (2, 7, "fp64", "BGK", cases.PERIODIC),
    (3, 8, "fp64", "BGK", cases.PERIODIC),
    (3, 9, "fp64", "TRT", CHANNEL),
    (2, 8, "fp64", "BGK", ("periodic", "periodic", "periodic", "periodic", "wall", "wall")),
    (3, 8, "fp32", "BGK", cases.PERIODIC),
    (2, 7, "fp16dev", "BGK", cases.PERIODIC),
])
def test_slabs_reproduce_the_undivided_box(parts, steps, storage, collision, faces):
    full = _full(steps, storage, collision, faces)
    g = _slabs(parts, steps, storage, collision, faces)
    try:
        f_full = full.populations().reshape(19, NZ, NY, NX)
        f_slab = np.concatenate([s.populations() for s in g.slabs], axis=1)
        assert f_slab.shape == f_full.shape
        assert rel_l2(f_slab, f_full) <= TOL[storage]
        for step in range(1, steps + 1):
            a, b = g.force(step), full.force(step)
            assert np.linalg.norm(a - b) <= 100 * TOL[storage] * np.linalg.norm(b) + 1e-12, (step, a, b)
        rho = np.concatenate([s.macros()[0] for s in g.slabs], axis=0)
        assert rel_l2(rho, full.macros()[0]) <= TOL[storage]
    finally:
        full.close()
        for s in g.slabs:
            s.close()


@pytest.mark.parametrize("parts,steps,collision,faces", [
    (2, 9, "BGK", cases.PERIODIC),
    (3, 10, "TRT", CHANNEL),
])
def test_slabs_match_the_oracle(gpu, oracle_lib, parts, steps, collision, faces):
    """The decomposed run against the CPU oracle of the whole box (FP64): owned-node
    populations, the summed force history and the density."""
    from oracle.oracle import OracleDomain

    o = OracleDomain(NX, NY, NZ, precision="fp64", **_kw("fp64", collision, faces))
    o.add_spheres(SPHERES)
    o.init_equilibrium()
    o.step(steps)
    g = _slabs(parts, steps, "fp64", collision, faces)
    try:
        f_slab = np.concatenate([s.populations() for s in g.slabs], axis=1)
        assert rel_l2(f_slab, o.populations().reshape(19, NZ, NY, NX)) <= 1e-12
        fs = np.stack([g.force(k) for k in range(1, steps + 1)])[:, :3]
        fo = o.force_history(1, steps)[:, :3]
        assert np.linalg.norm(fs - fo) <= 1e-9 * np.linalg.norm(fo) + 1e-11
        rho = np.concatenate([s.macros()[0] for s in g.slabs], axis=0)
        assert rel_l2(rho, o.macros()[0]) <= 1e-12
    finally:
        o.close()
        for s in g.slabs:
            s.close()


@pytest.mark.parametrize("storage,parts,steps", [("fp32", 2, 7), ("fp16dev", 3, 8), ("fp64", 2, 6)])
def test_slabs_on_the_pair_kernel(storage, parts, steps):
    """Periodic x and y with nx a multiple of 128: slabs run the pair kernel (FP32 and
    FP16-deviation) or the one-cell kernel without face handling (FP64), skipping their
    ghost planes block by block."""
    nx, ny, nz = 128, 12, 18
    xyzr = np.array([[20.5, 5.2, 9.1, 3.7], [70.2, 7.7, 0.8, 4.1], [101.3, 3.1, 12.2, 3.3]])
    kw = _kw(storage, "BGK", cases.PERIODIC)
    full = Domain(nx, ny, nz, **kw)
    full.add_spheres(xyzr)
    full.init_equilibrium()
    full.step(steps)
    slabs = [SlabDomain(nx, ny, nz, parts, r, **kw) for r in range(parts)]
    for s in slabs:
        s.add_spheres(xyzr)
        s.init_equilibrium()
    g = SlabGroup(slabs)
    g.step(steps)
    try:
        f_full = full.populations().reshape(19, nz, ny, nx)
        f_slab = np.concatenate([s.populations() for s in slabs], axis=1)
        assert rel_l2(f_slab, f_full) <= TOL[storage]
        a, b = g.force(steps), full.force(steps)
        assert np.linalg.norm(a - b) <= 100 * TOL[storage] * np.linalg.norm(b) + 1e-12, (a, b)
    finally:
        full.close()
        for s in slabs:
            s.close()


def test_halo_faces_are_checked():
    halo_x = ("halo", "halo") + ("periodic",) * 4
    with pytest.raises(LbmError):
        Domain(16, 8, 8, faces=halo_x)
    with pytest.raises(LbmError):
        Domain(16, 8, 2, faces=("periodic",) * 4 + ("halo", "halo"))
    d = Domain(16, 8, 8, faces=cases.PERIODIC)
    try:
        d.init_equilibrium()
        import torch

        buf = torch.empty(5 * 16 * 8 * 4, dtype=torch.uint8, device="cuda:0")
        assert d.halo_bytes == 0
        with pytest.raises(LbmError):
            d.halo_pack(0, buf)
    finally:
        d.close()
    s = SlabDomain(16, 8, 8, 2, 0)
    try:
        assert s.domain.halo_bytes == 5 * 16 * 8 * 4
        with pytest.raises(ValueError):
            s.add_body(abi.make_body(abi.BODY_SPHERE, (8, 4, 4), radius=2.0, moving=True))
        moving = abi.make_body(abi.BODY_SPHERE, (8, 4, 4), radius=2.0, moving=True)
        with pytest.raises(LbmError):
            s.domain.add_body(moving)
        s.init_equilibrium()
        with pytest.raises(LbmError):
            s.domain.halo_pack(2, buf)
    finally:
        s.close()
