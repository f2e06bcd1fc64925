"""GPU (liblbm3d.so through its C ABI) against the CPU oracle on the same inputs.

Tolerances: FP64 storage matches the FP64 oracle to rel. L2 1e-10 on rho/u and
1e-9 on forces (observed ~1e-14); flags and links are compared
bit-for-bit after every body move; FP32 reference mode is compared bit-for-bit
with the FP32 oracle (both avoid fused multiply-add and keep the reference's
operation order).
"""
import numpy as np
import pytest

from lbm3d_bb_b200 import Domain, abi
from oracle.oracle import OracleDomain
from tests import cases
from tests.cases import rel_l2

pytestmark = pytest.mark.gpu

TOL_FIELD = 1e-10
TOL_FORCE = 1e-9


def _force_close(fg, fo, tol):
    """rel. L2 with an absolute floor: the momentum exchange is a sum of O(1) terms
    that cancel to ~1e-15 when the force vanishes (equilibrium start)."""
    fg = np.asarray(fg, np.float64)
    fo = np.asarray(fo, np.float64)
    err = np.linalg.norm((fg - fo).ravel())
    assert err <= tol * np.linalg.norm(fo.ravel()) + 1e-11 * np.sqrt(fo.size), (err, np.linalg.norm(fo.ravel()))


def _macros_close(g, o, tol):
    for a, b in zip(g.macros(), o.macros()):
        assert rel_l2(a, b) <= tol, rel_l2(a, b)


@pytest.mark.parametrize("steps", [1, 2, 7, 40])
def test_sphere_channel_fp64(gpu, oracle_lib, steps):
    g = cases.sphere_channel(Domain)
    o = cases.sphere_channel(OracleDomain)
    g.step(steps)
    o.step(steps)
    assert rel_l2(g.populations(), o.populations()) <= 1e-12
    _macros_close(g, o, TOL_FIELD)
    fg = g.force_history(1, steps)
    fo = o.force_history(1, steps)
    _force_close(fg[:, :3], fo[:, :3], TOL_FORCE)
    assert abs(g.mass() - o.mass()) <= 1e-10 * abs(o.mass())


@pytest.mark.parametrize("outlet", ["pressure", "outflow"])
@pytest.mark.parametrize("storage_steps", [1, 2, 33])
def test_channel_outlets_fp64(gpu, oracle_lib, outlet, storage_steps):
    """Face nodes on the fast path (odd-sized box, non-periodic faces) against the oracle."""
    faces = ("inlet", outlet, "wall", "wall", "wall", "wall")
    kw = dict(nx=37, ny=19, nz=13, r=3.5, center=(12.2, 9.6, 6.4), u_in=0.05, faces=faces)
    g = cases.sphere_channel(Domain, **kw)
    o = cases.sphere_channel(OracleDomain, **kw)
    g.step(storage_steps)
    o.step(storage_steps)
    assert rel_l2(g.populations(), o.populations()) <= 1e-12
    _macros_close(g, o, TOL_FIELD)
    _force_close(g.force_history(1, storage_steps)[:, :3], o.force_history(1, storage_steps)[:, :3], TOL_FORCE)


def test_rotated_ellipsoid_channel_fp64(gpu, oracle_lib):
    """The warm-start workload's body: a rotated ellipsoid (flags and links bit-exact,
    fields and forces after 30 steps)."""
    import math

    a, b = 0.7, -1.1
    ca, sa, cb, sb = math.cos(a), math.sin(a), math.cos(b), math.sin(b)
    rz = np.array([[ca, -sa, 0], [sa, ca, 0], [0, 0, 1]])
    rx = np.array([[1, 0, 0], [0, cb, -sb], [0, sb, cb]])
    rot = (rz @ rx).ravel()
    faces = ("inlet", "pressure", "wall", "wall", "wall", "wall")

    def make(cls):
        d = cls(48, 24, 20, collision="BGK", storage="fp64", faces=faces, omega_p=1 / 0.7,
                face_u=cases.face_u_inlet(0.05))
        d.add_body(abi.make_body(abi.BODY_ELLIPSOID, (17.3, 11.8, 10.4), semi=(6.5, 3.2, 4.1), rot=rot))
        d.init_equilibrium()
        return d

    g, o = make(Domain), make(OracleDomain)
    for x, y in zip(g.flags(), o.flags()):
        assert np.array_equal(x, y)
    assert g.flags()[0].sum() > 200
    for x, y in zip(g.links(), o.links()):
        assert np.array_equal(x, y)
    g.step(30)
    o.step(30)
    assert rel_l2(g.populations(), o.populations()) <= 1e-12
    _force_close(g.force_history(1, 30)[:, :3], o.force_history(1, 30)[:, :3], TOL_FORCE)


def test_sphere_channel_flags_links(gpu, oracle_lib):
    g = cases.sphere_channel(Domain)
    o = cases.sphere_channel(OracleDomain)
    for a, b in zip(g.flags(), o.flags()):
        assert np.array_equal(a, b)
    for a, b in zip(g.links(), o.links()):
        assert np.array_equal(a, b)


def test_moving_sphere_trt_fp64(gpu, oracle_lib):
    g = cases.moving_sphere_trt(Domain)
    o = cases.moving_sphere_trt(OracleDomain)
    fresh_total = 0
    prev_solid = None
    for n in range(1, 61):
        pn, ph = cases.sphere_pose(g, n)
        g.update_body(pn, ph)
        o.update_body(pn, ph)
        ms_g, mb_g = g.flags()
        ms_o, mb_o = o.flags()
        assert np.array_equal(ms_g, ms_o), f"solid flags differ at step {n}"
        assert np.array_equal(mb_g, mb_o), f"boundary flags differ at step {n}"
        if n % 10 == 0:
            for a, b in zip(g.links(), o.links()):
                assert np.array_equal(a, b), f"links differ at step {n}"
        if prev_solid is not None:
            fresh_total += int(np.sum((prev_solid == 1) & (ms_g == 0)))
        prev_solid = ms_g
        g.step(1)
        o.step(1)
    assert fresh_total > 0, "the motion must uncover nodes for this test to exercise the refill"
    assert rel_l2(g.populations(), o.populations()) <= 1e-11
    _macros_close(g, o, TOL_FIELD)
    fg = g.force_history(1, 60)
    fo = o.force_history(1, 60)
    _force_close(fg[:, :3], fo[:, :3], TOL_FORCE)


@pytest.mark.parametrize("collision,accel", [("BGK", None), ("TRT", None), ("BGK", (1e-5, -4e-6, 3e-6)),
                                             ("TRT", (0.0, 2e-6, 1e-5))])
def test_porous_periodic_forcing_fp64(gpu, oracle_lib, collision, accel):
    """Guo forcing along x and along a general direction, BGK and TRT, against the oracle."""
    g = cases.porous_periodic(Domain, collision=collision, accel=accel)
    o = cases.porous_periodic(OracleDomain, collision=collision, accel=accel)
    assert np.array_equal(g.flags()[0], o.flags()[0])
    g.step(25)
    o.step(25)
    assert rel_l2(g.populations(), o.populations()) <= 1e-12
    _macros_close(g, o, TOL_FIELD)


# Stated bounds of the reduced-precision storage forms against the FP64 oracle on the
# miniature sphere channel (60 steps): rho and u (stacked velocity components) rel. L2,
# and the drag averaged over steps 41-60 (contract: drag within 0.5 % of FP64).
REDUCED = {"fp32": {"rho": 1e-6, "u": 1e-4, "drag": 1e-4},
           "fp16dev": {"rho": 1e-4, "u": 5e-3, "drag": 5e-3}}


@pytest.mark.parametrize("storage", ["fp32", "fp16dev"])
def test_reduced_precision_storage(gpu, oracle_lib, storage):
    tol = REDUCED[storage]
    g = cases.sphere_channel(Domain, storage=storage)
    o = cases.sphere_channel(OracleDomain)
    g.step(60)
    o.step(60)
    mg, mo = g.macros(), o.macros()
    e_rho = rel_l2(mg[0], mo[0])
    e_u = rel_l2(np.stack(mg[1:]), np.stack(mo[1:]))
    fd_g = g.force_history(41, 20)[:, 0].mean()
    fd_o = o.force_history(41, 20)[:, 0].mean()
    e_drag = abs(fd_g - fd_o) / abs(fd_o)
    print(f"\n[{storage} vs fp64 oracle] rho {e_rho:.3e} u {e_u:.3e} drag {e_drag:.3e}")
    assert e_rho <= tol["rho"]
    assert e_u <= tol["u"]
    assert e_drag <= tol["drag"]


def _ref_case(cls, precision_kw, coll="BGK", moving=True):
    nx, ny, nz = 40, 30, 3
    R, xc, yc = 4.16, 12.5, 15.5
    U = 0.075
    Re = 30.0
    nu = np.float32(U) * (np.float32(2.0) * np.float32(R)) / np.float32(Re)
    tau_p = np.float32(0.5) + np.float32(3.0) * nu
    tau_m = np.float32(0.5) + np.float32(0.1875) / (tau_p - np.float32(0.5))
    d = cls(nx, ny, nz, mode="reference", collision=coll, omega_p=float(np.float32(1.0) / tau_p),
            omega_m=float(np.float32(1.0) / tau_m), u_inf=(U, 0.0, 0.0), h=1.0, **precision_kw)
    d.add_body(abi.make_body(abi.BODY_CYLINDER_Z, (xc, yc, 0.0), radius=R, moving=moving))
    rng = np.random.default_rng(7)
    r = (2.0 * rng.random(d.N, dtype=np.float32) - 1.0).astype(np.float32)
    ux = (np.float32(U) * (np.float32(1.0) + np.float32(0.2) * r)).astype(np.float32)
    d.init_equilibrium(rho=np.ones(d.N), u=ux.astype(np.float64), v=np.zeros(d.N), w=np.zeros(d.N))
    return d


def _ref_pose(n):
    # MainCore.jl:72-80 law with a larger amplitude so nodes are uncovered quickly
    import math

    A, w = 1.7, 2.0 * math.pi / 50.0

    def at(t):
        y = np.float32(15.5 - A * math.sin(w * t))
        vy = np.float32(-A * w * math.cos(w * t))
        return y, vy

    y0, _ = at(n - 1.0)
    yh, vh = at(n - 0.5)
    pn = abi.make_pose(center=(12.5, float(y0), 0.0), cos_theta=1.0, sin_theta=0.0)
    ph = abi.make_pose(center=(12.5, float(yh), 0.0), vel=(0.0, float(vh), 0.0))
    return pn, ph


@pytest.mark.parametrize("coll", ["BGK", "TRT"])
def test_reference_mode_fp32_bit_exact(gpu, oracle_lib, coll):
    g = _ref_case(Domain, {"storage": "fp32"}, coll)
    o = _ref_case(OracleDomain, {"precision": "fp32"}, coll)
    assert np.array_equal(g.populations(np.float32), o.populations(np.float32))
    for n in range(1, 31):
        pn, ph = _ref_pose(n)
        g.update_body(pn, ph)
        o.update_body(pn, ph)
        for a, b in zip(g.flags(), o.flags()):
            assert np.array_equal(a, b), f"flags differ at step {n}"
        g.step(1)
        o.step(1)
        fg, fo = g.populations(np.float32), o.populations(np.float32)
        assert np.array_equal(fg, fo), f"populations differ at step {n}: max {np.abs(fg - fo).max()}"
    for a, b in zip(g.macros(np.float32), o.macros(np.float32)):
        assert np.array_equal(a, b)
    for a, b in zip(g.links(), o.links()):
        assert np.array_equal(a, b)
    fg = g.force_history(1, 30)
    fo = o.force_history(1, 30)
    _force_close(fg[:, :3], fo[:, :3], 1e-12)


def test_reference_mode_fp64(gpu, oracle_lib):
    g = _ref_case(Domain, {"storage": "fp64"}, "TRT")
    o = _ref_case(OracleDomain, {"precision": "fp64"}, "TRT")
    for n in range(1, 21):
        pn, ph = _ref_pose(n)
        g.update_body(pn, ph)
        o.update_body(pn, ph)
        g.step(1)
        o.step(1)
    assert rel_l2(g.populations(), o.populations()) <= 1e-13
    _macros_close(g, o, TOL_FIELD)
