"""Physics checks of the CPU oracle against analytic results (no reference output exists
to pin it; these tie its config-mode physics to known solutions)."""
import math

import numpy as np
import pytest

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
