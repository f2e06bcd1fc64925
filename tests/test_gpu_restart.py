"""Checkpoint and restart through the C ABI: populations exported after N steps
(lbm_get_populations, canonical layout) and loaded into a fresh context
(lbm_set_populations) continue exactly like the uninterrupted run — also when N is odd,
so that the restarted run takes its first step in the other AA phase."""
import numpy as np
import pytest

from lbm3d_bb_b200 import Domain
from tests import cases
from tests.cases import rel_l2

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-14, "fp32": 1e-7, "fp16dev": 1e-6}


def _porous(storage):
    return cases.porous_periodic(Domain, n=32, storage=storage, compute_force=True)


def _channel(storage):
    return cases.sphere_channel(Domain, storage=storage)


@pytest.mark.parametrize("make", [_porous, _channel], ids=["porous", "channel"])
@pytest.mark.parametrize("storage", ["fp64", "fp32", "fp16dev"])
@pytest.mark.parametrize("n_first", [7, 8])
def test_restart_continues_the_run(gpu, make, storage, n_first):
    m = 5
    whole = make(storage)
    first = make(storage)
    resumed = make(storage)
    try:
        whole.step(n_first + m)
        first.step(n_first)
        resumed.set_populations(first.populations())
        resumed.step(m)
        assert rel_l2(resumed.populations(), whole.populations()) <= TOL[storage]
        fa = whole.force_history(n_first + 1, m)
        fb = resumed.force_history(1, m)
        assert np.linalg.norm(fa - fb) <= 100 * TOL[storage] * np.linalg.norm(fa) + 1e-13
    finally:
        for d in (whole, first, resumed):
            d.close()
