"""Identical case set-ups for the GPU Domain and the CPU OracleDomain."""
from __future__ import annotations

import math

import numpy as np

from lbm3d_bb_b200 import abi

INLET_CHANNEL = ("inlet", "outflow", "wall", "wall", "wall", "wall")
PERIODIC = ("periodic",) * 6


def face_u_inlet(u):
    return [(u, 0.0, 0.0)] + [(0.0, 0.0, 0.0)] * 5


def sphere_channel(cls, nx=48, ny=24, nz=24, r=4.0, center=None, tau=0.8, u_in=0.04, storage="fp64",
                   faces=INLET_CHANNEL, **kw):
    """C1 in miniature: fixed sphere, equilibrium inlet, zero-gradient outlet, no-slip walls."""
    center = center or (nx / 4, ny / 2, nz / 2)
    d = cls(nx, ny, nz, collision="BGK", storage=storage, faces=faces, omega_p=1.0 / tau,
            face_u=face_u_inlet(u_in), **kw)
    d.add_sphere(center, r)
    d.init_equilibrium()
    return d


def moving_sphere_trt(cls, nx=64, ny=32, nz=32, r=5.0, tau_p=0.56, lam=3.0 / 16.0, u_in=0.03, amp=4.0,
                      period=200.0, storage="fp64", **kw):
    """C2 in miniature: TRT, oscillating sphere with fresh-node refill."""
    om_p = 1.0 / tau_p
    tau_m = 0.5 + lam / (tau_p - 0.5)
    d = cls(nx, ny, nz, collision="TRT", storage=storage, faces=INLET_CHANNEL, omega_p=om_p, omega_m=1.0 / tau_m,
            face_u=face_u_inlet(u_in), **kw)
    cx, cz = nx / 3.0, nz / 2.0
    d.add_body(abi.make_body(abi.BODY_SPHERE, (cx, ny / 2.0, cz), radius=r, moving=True))
    d.init_equilibrium()
    d._motion = (cx, ny / 2.0, cz, amp, period)
    return d


def sphere_pose(d, n):
    """Poses of step n (1-based): flags at t=n-1, kinematics at t=n-1/2."""
    cx, cy0, cz, amp, period = d._motion
    w = 2.0 * math.pi / period

    def at(t):
        y = cy0 + amp * math.sin(w * t)
        vy = amp * w * math.cos(w * t)
        return abi.make_pose(center=(cx, y, cz), vel=(0.0, vy, 0.0))

    return at(n - 1.0), at(n - 0.5)


def porous_periodic(cls, n=32, count=6, rmin=2.0, rmax=4.0, tau=0.6, g=1e-5, seed=3, storage="fp64",
                    accel=None, collision="BGK", **kw):
    """C3 in miniature: fully periodic box, random overlapping spheres, Guo body force
    (along x unless `accel` is given)."""
    rng = np.random.default_rng(seed)
    xyzr = np.concatenate([rng.uniform(0, n, (count, 3)), rng.uniform(rmin, rmax, (count, 1))], axis=1)
    if collision == "TRT":
        kw.setdefault("omega_m", 1.0 / (0.5 + 0.1875 / (tau - 0.5)))
    kw.setdefault("compute_force", False)
    d = cls(n, n, n, collision=collision, storage=storage, faces=PERIODIC, omega_p=1.0 / tau,
            accel=(g, 0.0, 0.0) if accel is None else accel, **kw)
    d.add_spheres(xyzr)
    d.init_equilibrium()
    return d


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.linalg.norm(b.ravel())
    return float(np.linalg.norm((a - b).ravel()) / (den if den > 0 else 1.0))
