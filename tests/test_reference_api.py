"""The Python mirror of the reference's module API (CPU semantics)."""
from pathlib import Path

import numpy as np
import pytest

from lbm3d_bb_b200 import reference_api as ra

GOLDEN = Path(__file__).resolve().parent / "golden"


def test_motion_at_is_float32_at_half_steps():
    law = ra.MotionLaw(lambda t: 3.0 * t, lambda t: 3.0, lambda t: t * t, lambda t: 2 * t, lambda t: 0.1,
                       lambda t: 0.0)
    p = ra.motion_at(5, np.float32(0.5), law, 0.5)
    t = (np.float32(4) + np.float32(0.5)) * np.float32(0.5)
    assert p["x_c"] == np.float32(3.0 * t) and p["y_c"] == np.float32(t * t)
    assert all(isinstance(v, np.float32) for v in p.values())


def test_errors_and_rank0_noops():
    with pytest.raises(ValueError, match="Unknown collision method: MRT"):
        ra.collision(None, None, *[None] * 9, 1.0, 1.0, "MRT", 10, 1)
    assert ra.collision(None, None, *[None] * 9, 1.0, 1.0, "BGK", 10, 0) is None  # master does nothing
    with pytest.raises(ValueError, match="Unknown or unimplemented boundary condition: MLS"):
        ra.solid_BC(None, None, None, None, None, None, None, None, None, None, "MLS", 1)
    assert ra.solid_BC(None, None, None, None, None, None, None, None, None, None, "MLS", 0) is None
    # both entries of the reference's dispatch table are accepted (IBB runs its SBB fallback)
    for bc in ("SBB", "IBB"):
        assert ra.solid_BC(None, None, None, None, None, None, None, None, None, None, bc, 1) is None
    assert ra.compute_aero(1, 1, 1, None, None, None, None, None, None, None, None, None, None, 1.0, None, 0) is None


def test_lattice_and_reference_area():
    p = ra.read_params_input(GOLDEN / "params_small_cylinder.txt")
    cx, cy, cz, w, bbopp = ra.gen_lattice_sets(p)
    assert list(bbopp) == [2, 1, 4, 3, 6, 5, 8, 7, 10, 9, 12, 11, 14, 13, 16, 15, 18, 17, 19]
    assert ra.ref_area_lat("CYL", p.R, p.chord, p.Nz, p.h) == np.float32(30.0)
    assert p.shape == "CYL" and p.coll == "BGK" and p.bc == "SBB" and p.n_save == 20


def test_main_core_law_matches_its_closed_form():
    p = ra.read_params_input(GOLDEN / "params_small_cylinder.txt")
    law = ra.main_core_law(p)
    Ae = np.float32(0.2) * np.float32(2) * p.R
    we = np.float32(2) * np.float32(np.pi) * (np.float32(0.154) * p.U_inf / (np.float32(2) * p.R))
    t = np.float32(17.5)
    assert law.y(t) == p.y_c - Ae * np.sin(we * t)
    assert law.ydot(t) == -Ae * we * np.cos(we * t)
