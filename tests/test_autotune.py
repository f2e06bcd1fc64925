"""Launch-shape autotuner: candidate shapes, choice of the fastest, and the JSON cache
(a stand-in domain and timer; the GPU test times a real domain)."""
import json

import numpy as np
import pytest

from lbm3d_bb_b200 import abi, autotune


class FakeDomain:
    def __init__(self, nx=96, ny=32, nz=32):
        self.cfg = abi.make_config(nx, ny, nz, faces=("inlet", "pressure", "wall", "wall", "wall", "wall"))
        self.shape = (nx, ny, nz)
        self.N = nx * ny * nz
        self.device = 0
        self.launch = None

    def set_launch(self, bx, by):
        assert bx * by <= 256 and (bx * by) % 32 == 0
        self.launch = (bx, by)


@pytest.mark.parametrize("nx", [9, 17, 32, 48, 96, 128, 512])
def test_candidates_are_valid_shapes(nx):
    c = autotune.candidates(nx)
    assert c
    for bx, by in c:
        assert bx * by <= 256 and (bx * by) % 32 == 0


def test_picks_fastest_and_caches(tmp_path, monkeypatch):
    monkeypatch.setenv("LBM3D_TUNE_CACHE", str(tmp_path / "shapes.json"))
    d = FakeDomain()
    cost = {(96, 2): 1.0, (64, 2): 0.7, (128, 1): 0.9}
    seen = []

    def timer():
        seen.append(d.launch)
        return cost.get(d.launch, 2.0)

    best = autotune.tune(d, shapes=list(cost), timer=timer, device_name="B200", save_state=False)
    assert best == (64, 2) and d.launch == (64, 2)
    assert sorted(seen) == sorted(cost)
    table = json.loads((tmp_path / "shapes.json").read_text())
    key = autotune.config_key(d, "B200")
    assert table[key]["best"] == [64, 2] and len(table[key]["ms_per_step"]) == 3
    # second call: cache hit, nothing timed
    d2 = FakeDomain()
    seen.clear()
    assert autotune.tune(d2, timer=timer, device_name="B200", save_state=False) == (64, 2)
    assert seen == [] and d2.launch == (64, 2)
    # another GPU or lattice is a different key
    assert autotune.config_key(d, "H100") != key
    assert autotune.config_key(FakeDomain(64, 32, 32), "B200") != key


@pytest.mark.gpu
def test_tune_real_domain_keeps_state(gpu, tmp_path, monkeypatch, oracle_lib):
    from lbm3d_bb_b200 import Domain
    from oracle.oracle import OracleDomain
    from tests import cases

    monkeypatch.setenv("LBM3D_TUNE_CACHE", str(tmp_path / "shapes.json"))
    d = cases.sphere_channel(Domain, nx=64, ny=24, nz=20)
    d.step(3)
    f0 = d.populations()
    bx, by = autotune.tune(d, steps=4, warmup=1)
    assert (bx * by) % 32 == 0 and d.launch() == (bx, by)
    assert np.array_equal(d.populations(), f0)  # the tuning steps are undone
    n = d.step_count
    d.step(10)
    o = cases.sphere_channel(OracleDomain, nx=64, ny=24, nz=20)
    o.set_populations(f0)
    o.step(10)
    assert cases.rel_l2(d.populations(), o.populations()) <= 1e-12
    assert d.step_count == n + 10
