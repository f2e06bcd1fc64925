"""The C++ oracle against the table-driven numpy transliteration of the reference.

Two independent restatements of the reference step — one by index arithmetic
(oracle/lbm_oracle.cpp), one replaying the reference's own list builders and
kernels in sequence (oracle/table_ref.py) — must agree bit for bit in FP32
(reference mode: virtual-fluid solids, moving cylinder, z-periodic, moving-wall
inlet/walls, anti-bounce-back outlet).  Neither could be pinned to reference
output (julia is absent), so this agreement is the strongest parity check
available for the restatement itself.
"""
import math

import numpy as np
import pytest

from lbm3d_bb_b200 import abi
from oracle.oracle import OracleDomain
from oracle.table_ref import TableReference


def _setup(coll, Nx=14, Ny=12, Nz=3, R=2.6, xc=5.5, yc=6.5, U=0.075, seed=11):
    h = 1.0
    Re = 20.0
    nu = np.float32(U) * (np.float32(2.0) * np.float32(R)) / np.float32(Re)
    tau_p = np.float32(0.5) + np.float32(3.0) * nu
    tau_m = np.float32(0.5) + np.float32(0.1875) / (tau_p - np.float32(0.5))
    om_p, om_m = float(np.float32(1.0) / tau_p), float(np.float32(1.0) / tau_m)
    N = Nx * Ny * Nz
    rng = np.random.default_rng(seed)
    r = (2.0 * rng.random(N, dtype=np.float32) - 1.0).astype(np.float32)
    ux = (np.float32(U) * (np.float32(1.0) + np.float32(0.2) * r)).astype(np.float32)
    t = TableReference(Nx, Ny, Nz, h=h, omega_p=om_p, omega_m=om_m, coll=coll, U_inf=U, R=R)
    t.init(np.ones(N, np.float32), ux, np.zeros(N, np.float32), np.zeros(N, np.float32))
    o = OracleDomain(Nx, Ny, Nz, precision="fp32", mode="reference", collision=coll, omega_p=om_p, omega_m=om_m,
                     u_inf=(U, 0.0, 0.0), h=h)
    o.add_body(abi.make_body(abi.BODY_CYLINDER_Z, (xc, yc, 0.0), radius=R, moving=True))
    o.init_equilibrium(rho=np.ones(N), u=ux.astype(np.float64), v=np.zeros(N), w=np.zeros(N))
    return t, o, (xc, yc)


def _poses(n, xc, yc):
    # MotionLaw of MainCore.jl:72-80 with a larger amplitude (uncovers nodes fast)
    A, w = np.float32(1.3), np.float32(2 * math.pi / 30.0)

    def at(tt):
        return np.float32(yc - A * np.sin(w * np.float32(tt))), np.float32(-A * w * np.cos(w * np.float32(tt)))

    y0, _ = at(n - 1.0)
    yh, vh = at(n - 0.5)
    return (np.float32(xc), y0), (np.float32(0.0), vh, np.float32(0.0), np.float32(xc), yh)


@pytest.mark.parametrize("coll", ["BGK", "TRT"])
def test_oracle_matches_table_transliteration_fp32(oracle_lib, coll):
    t, o, (xc, yc) = _setup(coll)
    N = t.N
    assert np.array_equal(o.populations(np.float32).T, t.f_old)
    for n in range(1, 13):
        pose_n, kin = _poses(n, xc, yc)
        pn = abi.make_pose(center=(float(pose_n[0]), float(pose_n[1]), 0.0), cos_theta=1.0, sin_theta=0.0)
        ph = abi.make_pose(center=(float(kin[3]), float(kin[4]), 0.0), vel=(float(kin[0]), float(kin[1]), 0.0),
                           omega=(0.0, 0.0, float(kin[2])))
        o.update_body(pn, ph)
        P, (ms, mb, ptr, lidx, dirs) = t.step(pose_n, kin)
        ms_o, mb_o = o.flags()
        assert np.array_equal(ms_o.astype(bool), ms), n
        assert np.array_equal(mb_o.astype(bool), mb), n
        optr, olidx, odirs = o.links()
        assert np.array_equal(optr, ptr) and np.array_equal(olidx, lidx) and np.array_equal(odirs, dirs), n
        o.step(1)
        fo = o.populations(np.float32).T
        assert np.array_equal(fo, t.f_old), f"step {n}: max |diff| {np.abs(fo - t.f_old).max()}"
        rho, u, v, w = o.macros(np.float32)
        assert np.array_equal(rho.ravel(), t.rho) and np.array_equal(u.ravel(), t.u)
        F = o.force(n)[:3]
        assert np.allclose(F, P, rtol=1e-12, atol=1e-13), (F, P)
    assert N == o.N
