"""D3Q27 (gen_lattice_sets q = 27, Utilities.jl:962-976) in reference mode against the CPU
oracle: the reference's step on the 27-velocity lattice (virtual-fluid solids, z-periodic
streaming, moving-wall inlet and walls, anti-bounce-back outlet, moving-wall bounce-back
on the moving cylinder), FP32 bit for bit after every step, FP64 to rounding; the
boundary flags and the link CSR with the corner directions; the interpolated
bounce-back; and main_simulation driven by a params.txt with q = 27."""
from pathlib import Path

import numpy as np
import pytest

from lbm3d_bb_b200 import Domain, abi
from lbm3d_bb_b200 import reference_api as ra
from oracle.oracle import OracleDomain
from tests.cases import rel_l2
from tests.test_gpu_parity import _ref_pose

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"


def _case(cls, precision_kw, coll="BGK", solid_bc="SBB"):
    nx, ny, nz = 40, 30, 4
    F = np.float32
    U, Re, R = 0.075, 30.0, 4.16
    nu = F(U) * (F(2.0) * F(R)) / F(Re)
    tau_p = F(0.5) + F(3.0) * nu
    tau_m = F(0.5) + F(0.1875) / (tau_p - F(0.5))
    d = cls(nx, ny, nz, mode="reference", collision=coll, omega_p=float(F(1.0) / tau_p),
            omega_m=float(F(1.0) / tau_m), u_inf=(U, 0.0, 0.0), h=1.0, q=27, solid_bc=solid_bc, **precision_kw)
    d.add_body(abi.make_body(abi.BODY_CYLINDER_Z, (12.5, 15.5, 0.0), radius=R, moving=True))
    rng = np.random.default_rng(27)
    r = (F(2) * rng.random(d.N, dtype=F) - F(1)).astype(F)
    ux = (F(U) * (F(1) + F(0.2) * r)).astype(F)
    d.init_equilibrium(rho=np.ones(d.N), u=ux.astype(np.float64), v=np.zeros(d.N), w=np.zeros(d.N))
    return d


@pytest.mark.parametrize("coll", ["BGK", "TRT"])
@pytest.mark.parametrize("solid_bc", ["SBB", "IBB"])
def test_d3q27_reference_mode_fp32_bit_exact(gpu, oracle_lib, coll, solid_bc):
    g = _case(Domain, {"storage": "fp32"}, coll, solid_bc)
    o = _case(OracleDomain, {"precision": "fp32"}, coll, solid_bc)
    try:
        assert g.populations(np.float32).shape == (27, g.N)
        assert np.array_equal(g.populations(np.float32), o.populations(np.float32))
        for n in range(1, 26):
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
        lg, lo = g.links(), o.links()
        for a, b in zip(lg, lo):
            assert np.array_equal(a, b)
        assert lg[2].max() > 18  # links along the corner directions
        fg, fo = g.force_history(1, 25)[:, :3], o.force_history(1, 25)[:, :3]
        assert np.linalg.norm(fg - fo) <= 1e-12 * np.linalg.norm(fo) + 1e-12
    finally:
        g.close()
        o.close()


def test_d3q27_reference_mode_fp64(gpu, oracle_lib):
    g = _case(Domain, {"storage": "fp64"}, "TRT")
    o = _case(OracleDomain, {"precision": "fp64"}, "TRT")
    try:
        for n in range(1, 21):
            pn, ph = _ref_pose(n)
            g.update_body(pn, ph)
            o.update_body(pn, ph)
            g.step(1)
            o.step(1)
        assert rel_l2(g.populations(), o.populations()) <= 1e-13
        for a, b in zip(g.macros(), o.macros()):
            assert rel_l2(a, b) <= 1e-10
        fg, fo = g.force_history(1, 20)[:, :3], o.force_history(1, 20)[:, :3]
        assert np.linalg.norm(fg - fo) <= 1e-9 * np.linalg.norm(fo) + 1e-11
    finally:
        g.close()
        o.close()


def test_d3q27_main_simulation_matches_oracle(gpu, oracle_lib):
    p = ra.read_params_input(GOLDEN / "params_d3q27.txt")
    assert p.q == 27
    res = ra.main_simulation(p, seed=5, macros_every_step=True)
    N = p.Nx * p.Ny * p.Nz
    o = OracleDomain(p.Nx, p.Ny, p.Nz, precision="fp32", mode="reference", collision=p.coll,
                     omega_p=float(p.omega_p), omega_m=float(p.omega_m), u_inf=(float(p.U_inf), 0.0, 0.0),
                     h=float(p.h), q=27)
    o.add_body(ra._shape_body(p))
    r = (np.float32(2) * np.random.default_rng(5).random(N, dtype=np.float32) - np.float32(1)).astype(np.float32)
    fac = np.float32(1) + np.float32(0.2) * r
    o.init_equilibrium(rho=np.ones(N), u=(p.U_inf * fac).astype(np.float64), v=np.zeros(N), w=np.zeros(N))
    law, bcs = ra.main_core_law(p), ra.SolidBCStruct()
    for n in range(1, p.n_max + 1):
        ra.motion(o, p.R, p.x_c, p.y_c, p.dt, p.h, bcs, law, n, 1)
        o.step(1)
    assert np.array_equal(res.domain.populations(np.float32), o.populations(np.float32))
    assert len(res.snapshots) == 2
    assert np.array_equal(res.snapshots[-1][1], o.macros(np.float32)[0].ravel())


def test_d3q27_rejected_in_config_mode(gpu):
    from lbm3d_bb_b200 import LbmError

    with pytest.raises(LbmError) as e:
        Domain(16, 8, 8, q=27)
    assert e.value.status == abi.LBM_ERR_UNSUPPORTED
