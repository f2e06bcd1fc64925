"""The bounded device waits give up and report, and the context keeps working.

Each library has one probe (lbm_wait_selftest, nn_wait_selftest): a single block waits
on an mbarrier that nothing arrives on and no copy or matrix multiply targets, through
the same bounded wait routine its pipelined kernels use, with a poll limit of a few
thousand instead of 2^22.  The wait runs out, the block records the failure in the
error word and returns with nothing in flight; the host reads a non-OK status.  A
normal step (or convolution) on the same context then runs and checks out."""
import numpy as np
import pytest

from lbm3d_bb_b200 import Domain, LbmError, abi
from oracle.oracle import OracleDomain
from tests import cases
from tests.cases import rel_l2

pytestmark = pytest.mark.gpu


def test_step_kernel_wait_gives_up_and_context_recovers(gpu, oracle_lib):
    g = cases.sphere_channel(Domain, nx=32, ny=16, nz=16, r=3.0)
    o = cases.sphere_channel(OracleDomain, nx=32, ny=16, nz=16, r=3.0)
    try:
        with pytest.raises(LbmError) as e:
            g._check(g._L.lbm_wait_selftest(g._h, 4096))
        assert e.value.status == abi.LBM_ERR_TIMEOUT
        assert "gave up" in str(e.value)
        g.synchronize()  # the error word was cleared when it was reported
        g.step(5)
        o.step(5)
        g.synchronize()
        assert rel_l2(g.populations(), o.populations()) <= 1e-12
        g.check_finite()
    finally:
        g.close()
        o.close()


def test_selftest_rejects_limits_outside_range(gpu):
    d = Domain(16, 8, 8, storage="fp32")
    try:
        for polls in (0, -3, (1 << 22) + 1):
            with pytest.raises(LbmError) as e:
                d._check(d._L.lbm_wait_selftest(d._h, polls))
            assert e.value.status == abi.LBM_ERR_ARG
    finally:
        d.close()


def test_tcgen05_wait_gives_up_and_convolution_recovers(gpu):
    import torch

    from lbm3d_bb_b200 import unet as N
    from oracle import unet_ref as U

    assert N.lib().nn_wait_selftest(4096, None) != 0
    assert b"gave up" in (N.lib().nn_last_error() or b"")
    N.tc_status()  # cleared: no error pending
    prev = N.set_conv_engine("tcgen05")
    try:
        ops = N.Ops()
        shape, cin, cout = (1, 2, 4, 32), 16, 32
        rng = np.random.default_rng(5)
        x = U.to_bf16(rng.standard_normal(shape + (cin,)))
        w = U.to_bf16(rng.standard_normal((27, cout, cin)) / np.sqrt(27 * cin))
        b = rng.standard_normal(cout) * 0.1

        def dev(a, bf16=True):
            t = torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()
            if not bf16:
                return t
            out = torch.empty(t.shape, dtype=torch.bfloat16, device="cuda")
            ops.to_bf16(t, out)
            return out

        y = torch.empty(shape + (cout,), dtype=torch.bfloat16, device="cuda")
        ops.conv(dev(x), dev(w), dev(b, False), y, shape, cin, cout, False)
        N.tc_status()
        f = torch.empty(y.shape, dtype=torch.float32, device="cuda")
        ops.from_bf16(y, f)
        torch.cuda.synchronize()
        got = f.cpu().numpy().astype(np.float64)
        ref = U.conv(x, w, b)
        assert rel_l2(got, ref) <= 1e-2
    finally:
        N.set_conv_engine(prev)
