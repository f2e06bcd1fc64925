"""main_simulation (MainCore.jl's loop over the mirror API) on the GPU against the
oracle driven through the same motion/initialisation calls."""
from pathlib import Path

import numpy as np
import pytest

from lbm3d_bb_b200 import abi
from lbm3d_bb_b200 import reference_api as ra
from oracle.oracle import OracleDomain

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"


# params_default_reduced.txt is the reference's shipped input (input/params.txt: cylinder
# R = 16.16, Re = 185, U_inf = 0.075, BC IBB, BGK) on a 241 x 161 x 3 box for 60 steps.
@pytest.mark.parametrize("params_file", ["params_small_cylinder.txt", "params_default_reduced.txt"])
def test_main_simulation_matches_oracle(gpu, oracle_lib, params_file):
    p = ra.read_params_input(GOLDEN / params_file)
    res = ra.main_simulation(p, seed=3, macros_every_step=True)
    # the oracle, fed the same initial field and the same motion! calls
    N = p.Nx * p.Ny * p.Nz
    o = OracleDomain(p.Nx, p.Ny, p.Nz, precision="fp32", mode="reference", collision=p.coll,
                     omega_p=float(p.omega_p), omega_m=float(p.omega_m), u_inf=(float(p.U_inf), 0.0, 0.0),
                     h=float(p.h))
    o.add_body(ra._shape_body(p))
    r = (np.float32(2) * np.random.default_rng(3).random(N, dtype=np.float32) - np.float32(1)).astype(np.float32)
    fac = np.float32(1) + np.float32(0.2) * r
    o.init_equilibrium(rho=np.ones(N), u=(p.U_inf * fac).astype(np.float64), v=np.zeros(N), w=np.zeros(N))
    law = ra.main_core_law(p)
    bcs = ra.SolidBCStruct()
    fc = np.float32(1) / (np.float32(0.5) * p.rho_inf * (p.U_inf * p.U_inf) *
                          ra.ref_area_lat(p.shape, p.R, p.chord, p.Nz, p.h))
    CD = np.zeros(p.n_max, np.float32)
    for n in range(1, p.n_max + 1):
        ra.motion(o, p.R, p.x_c, p.y_c, p.dt, p.h, bcs, law, n, 1)
        o.step(1)
        CD[n - 1] = np.float32(o.force(n)[0]) * fc
    g = res.domain
    assert np.array_equal(g.populations(np.float32), o.populations(np.float32))
    assert np.allclose(res.CD, CD, rtol=1e-6, atol=1e-9)
    assert len(res.snapshots) == 2 and res.snapshots[-1][0] == p.n_max
    rho_o, u_o, _, _ = o.macros(np.float32)
    assert np.array_equal(res.snapshots[-1][1], rho_o.ravel())
    assert np.array_equal(res.snapshots[-1][2], u_o.ravel())
    assert res.mlups > 0
