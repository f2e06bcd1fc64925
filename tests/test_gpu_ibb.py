"""Interpolated bounce-back (lbm_config.solid_bc = LBM_SOLID_IBB, reference mode) against
the CPU oracle.

The rule is IBB!_gpu (SolidBC.jl:253-338) as it is meant to work: q from phi at the two
ends of each link, the wall at x_b + q c, the fluid-side neighbour for q <= 1/2.  The
GPU and the oracle evaluate the FP32 geometry with the same operations (no fused
multiply-add on either side), so FP32 populations agree bit for bit after every step
of a moving body; FP64 agrees to rounding.  Bodies: the reference's cylinder and a
cambered NACA band at an angle of attack (its concave lower surface gives links whose
phi changes sign on either side of x_b)."""
import math

import numpy as np
import pytest

from lbm3d_bb_b200 import Domain, abi
from oracle.oracle import OracleDomain
from tests.cases import rel_l2

pytestmark = pytest.mark.gpu


def _case(cls, shape, solid_bc="IBB", **kw):
    nx, ny, nz = 64, 40, 3
    U, Re = 0.05, 30.0
    F = np.float32
    L = F(8.32) if shape == "cyl" else F(24.0)
    nu = F(U) * L / F(Re)
    tau_p = F(0.5) + F(3.0) * nu
    tau_m = F(0.5) + F(0.1875) / (tau_p - F(0.5))
    d = cls(nx, ny, nz, mode="reference", collision=kw.pop("coll", "BGK"), omega_p=float(F(1.0) / tau_p),
            omega_m=float(F(1.0) / tau_m), u_inf=(U, 0.0, 0.0), h=1.0, solid_bc=solid_bc, **kw)
    if shape == "cyl":
        body = abi.make_body(abi.BODY_CYLINDER_Z, (20.5, 20.3, 0.0), radius=4.16, moving=True)
    else:  # NACA 4412, chord 24, pivot at the quarter chord
        body = abi.make_body(abi.BODY_NACA_Z, (24.0, 20.2, 0.0), moving=True, chord=24.0,
                             naca=(float(F(0.04)), float(F(0.4)), float(F(0.12))), x_int=float(F(1.0089304)),
                             x_le_offset=float(F(0.25) * F(24.0)))
    d.add_body(body)
    rng = np.random.default_rng(9)
    r = (F(2) * rng.random(d.N, dtype=F) - F(1)).astype(F)
    ux = (F(U) * (F(1) + F(0.2) * r)).astype(F)
    d.init_equilibrium(rho=np.ones(d.N), u=ux.astype(np.float64), v=np.zeros(d.N), w=np.zeros(d.N))
    return d


def _pose(shape, n):
    """Heave (and, for the airfoil, pitch about 8 degrees) at t = n-1 and n-1/2; the body
    moves at most 0.03 lattice units per step."""
    F = np.float32
    A, w = 1.3, 2.0 * math.pi / 300.0
    yc0 = 20.3 if shape == "cyl" else 20.2
    xc = 20.5 if shape == "cyl" else 24.0

    def at(t):
        y = F(yc0 - A * math.sin(w * t))
        vy = F(-A * w * math.cos(w * t))
        th = F(0.0) if shape == "cyl" else F(-math.radians(8.0) + 0.05 * math.sin(w * t))
        om = F(0.0) if shape == "cyl" else F(0.05 * w * math.cos(w * t))
        return y, vy, th, om

    y0, _, th0, _ = at(n - 1.0)
    yh, vh, thh, omh = at(n - 0.5)
    pn = abi.make_pose(center=(xc, float(y0), 0.0), cos_theta=float(F(math.cos(th0))), sin_theta=float(F(math.sin(th0))))
    ph = abi.make_pose(center=(xc, float(yh), 0.0), cos_theta=float(F(math.cos(thh))),
                       sin_theta=float(F(math.sin(thh))), vel=(0.0, float(vh), 0.0), omega=(0.0, 0.0, float(omh)))
    return pn, ph


@pytest.mark.parametrize("shape", ["cyl", "naca"])
@pytest.mark.parametrize("coll", ["BGK", "TRT"])
def test_interpolated_bb_fp32_bit_exact(gpu, oracle_lib, shape, coll):
    g = _case(Domain, shape, storage="fp32", coll=coll)
    o = _case(OracleDomain, shape, precision="fp32", coll=coll)
    try:
        for n in range(1, 31):
            pn, ph = _pose(shape, n)
            g.update_body(pn, ph)
            o.update_body(pn, ph)
            g.step(1)
            o.step(1)
            fg, fo = g.populations(np.float32), o.populations(np.float32)
            assert np.array_equal(fg, fo), f"step {n}: max |diff| {np.abs(fg - fo).max()}"
        fgh, foh = g.force_history(1, 30)[:, :3], o.force_history(1, 30)[:, :3]
        assert np.linalg.norm(fgh - foh) <= 1e-12 * np.linalg.norm(foh) + 1e-12
        assert np.abs(foh[:, 0]).max() > 0.0
    finally:
        g.close()
        o.close()


@pytest.mark.parametrize("shape", ["cyl", "naca"])
def test_interpolated_bb_fp64(gpu, oracle_lib, shape):
    g = _case(Domain, shape, storage="fp64")
    o = _case(OracleDomain, shape, precision="fp64")
    try:
        for n in range(1, 21):
            pn, ph = _pose(shape, n)
            g.update_body(pn, ph)
            o.update_body(pn, ph)
            g.step(1)
            o.step(1)
        assert rel_l2(g.populations(), o.populations()) <= 1e-13
        fg, fo = g.force_history(1, 20)[:, :3], o.force_history(1, 20)[:, :3]
        assert np.linalg.norm(fg - fo) <= 1e-10 * np.linalg.norm(fo) + 1e-12
    finally:
        g.close()
        o.close()


def test_interpolated_bb_differs_from_sbb_and_stays_close(gpu):
    """The interpolation changes the populations next to the wall (it is not the SBB
    rule under another name) while the drag stays within a few per cent of SBB's."""
    runs = {}
    for bc in ("SBB", "IBB"):
        d = _case(Domain, "cyl", solid_bc=bc, storage="fp64")
        for n in range(1, 201):
            d.update_body(*_pose("cyl", n))
            d.step(1)
        runs[bc] = (d.populations(), d.force_history(101, 100)[:, 0].mean())
        d.close()
    assert rel_l2(runs["IBB"][0], runs["SBB"][0]) > 1e-6
    assert abs(runs["IBB"][1] - runs["SBB"][1]) <= 0.1 * abs(runs["SBB"][1])


def test_interpolated_bb_rejected_outside_reference_mode(gpu):
    from lbm3d_bb_b200 import LbmError

    with pytest.raises(LbmError) as e:
        Domain(16, 8, 8, solid_bc="IBB")
    assert e.value.status == abi.LBM_ERR_UNSUPPORTED
