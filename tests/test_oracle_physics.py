"""Checks of the CPU oracle against analytic results and definitions (no reference output
exists to pin it): config-mode physics against known solutions, and the reference-mode
bounce-back mask and link CSR against a brute-force evaluation of their definitions."""
import math

import numpy as np
import pytest

from lbm3d_bb_b200 import abi
from oracle.oracle import OracleDomain
from tests import cases


def test_mass_conserved_periodic_fp64(oracle_lib):
    n = 12
    rng = np.random.default_rng(0)
    N = n ** 3
    d = OracleDomain(n, n, n, faces=cases.PERIODIC, omega_p=1.6, compute_force=False)
    d.init_equilibrium(rho=1 + 0.01 * rng.standard_normal(N), u=0.02 * rng.standard_normal(N),
                       v=0.02 * rng.standard_normal(N), w=0.02 * rng.standard_normal(N))
    m0 = d.mass()
    d.step(40)
    assert abs(d.mass() - m0) <= 1e-12 * m0


def test_rest_state_is_fixed_point(oracle_lib):
    d = cases.sphere_channel(OracleDomain, u_in=0.0)
    f0 = d.populations()
    d.step(5)
    assert np.max(np.abs(d.populations() - f0)) < 1e-15


def test_taylor_green_decay_rate(oracle_lib):
    n, tau, U = 32, 0.8, 0.01
    nu = (tau - 0.5) / 3.0
    x = np.arange(n) + 0.5
    X, Y = np.meshgrid(x, x, indexing="xy")  # (y, x)
    k = 2 * np.pi / n
    ux = U * np.sin(k * X) * np.cos(k * Y)
    uy = -U * np.cos(k * X) * np.sin(k * Y)
    nz = 2
    u3 = np.broadcast_to(ux, (nz, n, n)).ravel()
    v3 = np.broadcast_to(uy, (nz, n, n)).ravel()
    d = OracleDomain(n, n, nz, faces=cases.PERIODIC, omega_p=1 / tau, compute_force=False)
    d.init_equilibrium(rho=None, u=u3, v=v3, w=np.zeros_like(u3))
    T = 200
    d.step(T)
    _, u, _, _ = d.macros()
    amp = np.sum(u[0] * ux) / np.sum(ux * ux)
    expect = math.exp(-2 * nu * k * k * T)
    assert abs(amp - expect) / expect < 0.01, (amp, expect)


def test_poiseuille_profile_under_body_force(oracle_lib):
    ny, g, tau = 16, 1e-6, 1.0
    nu = (tau - 0.5) / 3.0
    d = OracleDomain(4, ny, 2, faces=("periodic", "periodic", "wall", "wall", "periodic", "periodic"),
                     omega_p=1 / tau, accel=(g, 0.0, 0.0), compute_force=False)
    d.init_equilibrium()
    d.step(4000)
    _, u, _, _ = d.macros()
    y = np.arange(ny) + 0.5
    exact = g / (2 * nu) * y * (ny - y)  # half-way bounce-back walls at y = 0 and y = ny
    prof = u[0, :, 0]
    assert np.max(np.abs(prof - exact)) / exact.max() < 0.01


def test_trt_equals_bgk_when_rates_match(oracle_lib):
    a = cases.sphere_channel(OracleDomain, tau=0.8)
    b = OracleDomain(48, 24, 24, collision="TRT", faces=cases.INLET_CHANNEL, omega_p=1 / 0.8, omega_m=1 / 0.8,
                     face_u=cases.face_u_inlet(0.04))
    b.add_sphere((12.0, 12.0, 12.0), 4.0)
    b.init_equilibrium()
    a.step(15)
    b.step(15)
    assert cases.rel_l2(a.populations(), b.populations()) < 1e-13


def test_centred_sphere_has_no_lift_or_side_force(oracle_lib):
    d = cases.sphere_channel(OracleDomain)
    d.step(60)
    F = d.force()
    assert F[0] > 0
    assert abs(F[1]) < 1e-10 * F[0] and abs(F[2]) < 1e-10 * F[0]


@pytest.mark.parametrize("coll", ["BGK", "TRT"])
def test_reference_mode_evolves_solid_nodes_as_virtual_fluid(oracle_lib, coll):
    """Reference quirk: solid nodes are collided and streamed (Collision.jl:227-228)."""
    from lbm3d_bb_b200 import abi

    d = OracleDomain(20, 16, 3, mode="reference", collision=coll, omega_p=1.2, omega_m=1.1, u_inf=(0.05, 0, 0))
    d.add_body(abi.make_body(abi.BODY_CYLINDER_Z, (8.0, 8.0, 0.0), radius=3.0))
    d.init_equilibrium(u=np.full(d.N, 0.05))
    f0 = d.populations()
    d.step(3)
    ms, _ = d.flags()
    solid = np.flatnonzero(ms)
    assert solid.size > 0
    assert np.max(np.abs(d.populations()[:, solid] - f0[:, solid])) > 1e-6


def _brute_force_links(ms, shape, cxyz):
    """mask_bb and the link CSR by their definitions (Geometry.jl:122-148, 181-262):
    a fluid node is a bounce-back node when a neighbour inside the box (no wrap, as in
    the reference's neighbour table, Utilities.jl:555-570) is solid; its links are those
    directions, ascending, 1-based; bb_ptr is 1-based with bb_ptr[1] = 1."""
    nx, ny, nz = shape
    solid = ms.reshape(nz, ny, nx).astype(bool)
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    hit = np.zeros((19, nz, ny, nx), bool)
    for q in range(19):
        jx, jy, jz = x + cxyz[0][q], y + cxyz[1][q], z + cxyz[2][q]
        inside = (jx >= 0) & (jx < nx) & (jy >= 0) & (jy < ny) & (jz >= 0) & (jz < nz)
        s = np.zeros_like(inside)
        s[inside] = solid[jz[inside], jy[inside], jx[inside]]
        hit[q] = s & ~solid
    mb = hit.any(axis=0).ravel()
    h = hit.reshape(19, -1)
    counts = h.sum(axis=0).astype(np.int64)
    ptr = np.concatenate([[1], 1 + np.cumsum(counts)]).astype(np.int32)
    node, = np.nonzero(counts)
    lidx = np.repeat(node + 1, counts[node]).astype(np.int32)
    dirs = np.concatenate([np.nonzero(h[:, a])[0] + 1 for a in node]).astype(np.int8) if len(node) else \
        np.zeros(0, np.int8)
    return mb, ptr, lidx, dirs


@pytest.mark.parametrize("body", ["cylinder", "naca"])
def test_link_csr_matches_its_definition(oracle_lib, body):
    """The oracle's mask_bb and link CSR (the bit-exact contract the GPU tests hold the
    kernels to) against a brute-force evaluation of the reference's definitions."""
    from lbm3d_bb_b200.domain import lattice

    cx, cy, cz, _, _ = lattice()
    nx, ny, nz = 40, 24, 3
    d = OracleDomain(nx, ny, nz, mode="reference", collision="BGK", omega_p=1.2, u_inf=(0.05, 0, 0))
    if body == "cylinder":
        d.add_body(abi.make_body(abi.BODY_CYLINDER_Z, (14.3, 12.1, 0.0), radius=5.2))
    else:
        d.add_body(abi.make_body(abi.BODY_NACA_Z, (16.0, 12.0, 0.0), chord=18.0, naca=(0.02, 0.4, 0.12)))
    d.init_equilibrium()
    ms, mb = d.flags()
    ptr, lidx, dirs = d.links()
    assert ms.sum() > 0
    mb_ref, ptr_ref, lidx_ref, dirs_ref = _brute_force_links(ms, (nx, ny, nz), (cx, cy, cz))
    assert np.array_equal(mb.astype(bool), mb_ref)
    assert np.array_equal(ptr, ptr_ref)
    assert np.array_equal(lidx, lidx_ref)
    assert np.array_equal(dirs, dirs_ref)


@pytest.mark.parametrize("shape", ["cyl", "naca"])
def test_interpolated_bounce_back_keeps_the_rest_state(oracle_lib, shape):
    """With every f* at its rest value w_d both interpolation branches of the interpolated
    bounce-back return w_d (2q w + (1-2q) w, w/(2q) + (1 - 1/(2q)) w), so a fluid and body
    at rest stay at rest; the same run with a uniform stream is finite and differs from SBB."""
    F = np.float32

    def make(bc, U):
        d = OracleDomain(48, 32, 3, precision="fp64", mode="reference", collision="BGK", omega_p=1.4,
                         u_inf=(U, 0.0, 0.0), h=1.0, solid_bc=bc)
        if shape == "cyl":
            d.add_body(abi.make_body(abi.BODY_CYLINDER_Z, (16.5, 16.3, 0.0), radius=5.3, moving=True))
        else:
            d.add_body(abi.make_body(abi.BODY_NACA_Z, (20.0, 16.2, 0.0), moving=True, chord=20.0,
                                     naca=(float(F(0.04)), float(F(0.4)), float(F(0.12))),
                                     x_int=float(F(1.0089304)), x_le_offset=float(F(0.25) * F(20.0))))
        d.init_equilibrium(rho=np.ones(d.N), u=np.full(d.N, U), v=np.zeros(d.N), w=np.zeros(d.N))
        th = -math.radians(6.0) if shape == "naca" else 0.0
        pose = abi.make_pose(center=(16.5 if shape == "cyl" else 20.0, 16.3 if shape == "cyl" else 16.2, 0.0),
                             theta=th)
        d.update_body(pose, pose)
        return d

    d = make("IBB", 0.0)
    f0 = d.populations()
    d.step(6)
    assert np.max(np.abs(d.populations() - f0)) < 1e-15
    a, b = make("IBB", 0.05), make("SBB", 0.05)
    a.step(20)
    b.step(20)
    fa, fb = a.populations(), b.populations()
    assert np.all(np.isfinite(fa))
    assert np.max(np.abs(fa - fb)) > 1e-8
