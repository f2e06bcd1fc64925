"""Numerical watchdogs through the C ABI: the FP64 mass sum (lbm_mass) stays constant on
a closed periodic box, and a non-finite value injected from the host into one domain of
a batched sweep is reported by lbm_check for that domain only (the fault is a value,
injected through lbm_set_populations: nothing faults or stalls the GPU)."""
import numpy as np
import pytest

from lbm3d_bb_b200 import Domain, LbmError
from lbm3d_bb_b200.batch import Batch
from tests import cases
from tests.test_gpu_batch import _members

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("storage,tol", [("fp64", 1e-12), ("fp32", 1e-6), ("fp16dev", 1e-4)])
def test_mass_is_conserved_on_a_closed_box(gpu, storage, tol):
    d = cases.porous_periodic(Domain, n=32, storage=storage)  # body force: flow, no mass source
    try:
        m0 = d.mass()
        d.step(40)
        assert abs(d.mass() - m0) <= tol * m0
        d.check_finite()
    finally:
        d.close()


def test_nan_in_one_domain_is_reported_for_that_domain(gpu):
    doms = _members(Domain, "fp32")
    bad = 2
    try:
        f = doms[bad].populations()
        solid = doms[bad].flags()[0]
        node = int(np.flatnonzero(solid == 0)[len(np.flatnonzero(solid == 0)) // 2])  # a fluid node
        f[5, node] = np.nan
        doms[bad].set_populations(f)
        with Batch(doms) as b:
            b.step(4)
            b.synchronize()
        for k, d in enumerate(doms):
            if k == bad:
                with pytest.raises(LbmError):
                    d.check_finite()
            else:
                d.check_finite()
    finally:
        for d in doms:
            d.close()
