"""The warm-start network's kernels (libunet3d.so) against the CPU restatement
(oracle/unet_ref.py): each layer type, then a whole forward/backward pass.

The GPU stores activations and working weights in BF16 and accumulates in FP32; the
oracle rounds to BF16 at the same places and accumulates in FP64, so results agree
to a few BF16 ulps where a stored value sits next to a rounding boundary (stated
per check).  FP32 outputs (weight gradients) agree to FP32 summation error."""
import numpy as np
import pytest

from lbm3d_bb_b200 import unet as N
from oracle import unet_ref as U
from tests.cases import rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ops(gpu):
    return N.Ops()


def _dev(a, ops, bf16=True):
    import torch

    t = torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()
    if not bf16:
        return t
    b = torch.empty(t.shape, dtype=torch.bfloat16, device="cuda")
    ops.to_bf16(t, b)
    return b


def _host(t, ops):
    import torch

    if t.dtype == torch.bfloat16:
        f = torch.empty(t.shape, dtype=torch.float32, device="cuda")
        ops.from_bf16(t, f)
        t = f
    torch.cuda.synchronize()
    return t.cpu().numpy().astype(np.float64)


SHAPE = (2, 3, 5, 32)


@pytest.fixture(params=["mma", "tcgen05", "auto", "tcgen05-tma"])
def engine(request, gpu):
    prev = N.set_conv_engine(request.param)
    yield request.param
    N.tc_status()
    N.set_conv_engine(prev)


@pytest.mark.parametrize("cin,cout", [(16, 16), (16, 32), (32, 64), (64, 64), (96, 32), (48, 16), (32, 48), (64, 96)])
@pytest.mark.parametrize("relu", [False, True])
def test_conv_forward(ops, engine, cin, cout, relu):
    import torch

    rng = np.random.default_rng(cin * 1000 + cout)
    x = U.to_bf16(rng.standard_normal(SHAPE + (cin,)))
    w = U.to_bf16(rng.standard_normal((27, cout, cin)) / np.sqrt(27 * cin))
    b = rng.standard_normal(cout) * 0.1
    y = torch.empty(SHAPE + (cout,), dtype=torch.bfloat16, device="cuda")
    ops.conv(_dev(x, ops), _dev(w, ops), _dev(b, ops, False), y, SHAPE, cin, cout, relu)
    ref = U.conv(x, w, b)
    if relu:
        ref = np.maximum(ref, 0)
    got = _host(y, ops)
    assert rel_l2(got, U.to_bf16(ref)) <= 3e-3  # BF16 output rounding of FP32 vs FP64 sums
    assert rel_l2(got, ref) <= 5e-3


@pytest.mark.parametrize("shape", [(2, 3, 8, 32), (1, 2, 2, 128), (1, 2, 4, 64), (1, 3, 16, 16), (1, 2, 3, 256)])
@pytest.mark.parametrize("cin,cout", [(16, 32), (32, 64), (96, 32), (16, 96), (48, 48), (64, 16)])
def test_conv_forward_tma_fed(ops, shape, cin, cout):
    """Shapes whose 128-voxel tiles are whole rows or part of one row take the TMA-fed
    tcgen05 kernel (halo from the copy engine's zero fill)."""
    import torch

    prev = N.set_conv_engine("tcgen05-tma")
    try:
        assert N.lib().nn_conv_uses_tma(shape[2], shape[3], cin, cout) == 1
        rng = np.random.default_rng(sum(shape) + cin + cout)
        x = U.to_bf16(rng.standard_normal(shape + (cin,)))
        w = U.to_bf16(rng.standard_normal((27, cout, cin)) / np.sqrt(27 * cin))
        b = rng.standard_normal(cout) * 0.1
        y = torch.empty(shape + (cout,), dtype=torch.bfloat16, device="cuda")
        ops.conv(_dev(x, ops), _dev(w, ops), _dev(b, ops, False), y, shape, cin, cout, True)
        N.tc_status()
        ref = np.maximum(U.conv(x, w, b), 0)
        assert rel_l2(_host(y, ops), ref) <= 5e-3
    finally:
        N.set_conv_engine(prev)


@pytest.mark.parametrize("cin,cout", [(16, 16), (32, 16), (48, 16), (96, 32), (16, 32), (32, 64), (64, 64)])
def test_conv_weight_and_bias_gradient(ops, cin, cout):
    import torch

    rng = np.random.default_rng(7 + cin + cout)
    x = U.to_bf16(rng.standard_normal(SHAPE + (cin,)))
    dy = U.to_bf16(rng.standard_normal(SHAPE + (cout,)))
    w = np.zeros((27, cout, cin))
    _, dw_ref, db_ref = U.conv_bwd(x, w, dy)
    dw = torch.zeros((27, cout, cin), dtype=torch.float32, device="cuda")
    db = torch.zeros(cout, dtype=torch.float32, device="cuda")
    dyd = _dev(dy, ops)
    ops.bwd_weight(_dev(x, ops), dyd, dw, SHAPE, cin, cout)
    ops.bias_grad(dyd, db, int(np.prod(SHAPE)), cout)
    assert rel_l2(_host(dw, ops), dw_ref) <= 1e-5
    assert rel_l2(_host(db, ops), db_ref) <= 1e-5


def test_conv_weight_gradient_many_chunks(ops):
    """More voxels than one block's chunk: partial sums of several blocks add up."""
    import torch

    shape = (2, 20, 16, 32)  # 20480 voxels = 5 chunks of 4096
    rng = np.random.default_rng(3)
    x = U.to_bf16(rng.standard_normal(shape + (16,)))
    dy = U.to_bf16(rng.standard_normal(shape + (32,)))
    _, dw_ref, _ = U.conv_bwd(x, np.zeros((27, 32, 16)), dy)
    dw = torch.zeros((27, 32, 16), dtype=torch.float32, device="cuda")
    ops.bwd_weight(_dev(x, ops), _dev(dy, ops), dw, shape, 16, 32)
    assert rel_l2(_host(dw, ops), dw_ref) <= 1e-5


@pytest.mark.parametrize("cin,cout", [(16, 16), (16, 32), (32, 64), (96, 32), (48, 16)])
def test_conv_data_gradient(ops, engine, cin, cout):
    import torch

    rng = np.random.default_rng(11 + cin + cout)
    x = np.zeros(SHAPE + (cin,))
    w = U.to_bf16(rng.standard_normal((27, cout, cin)) / np.sqrt(27 * cin))
    dy = U.to_bf16(rng.standard_normal(SHAPE + (cout,)))
    dx_ref, _, _ = U.conv_bwd(x, w, dy)
    wd = _dev(w, ops)
    wt = torch.empty((27, cin, cout), dtype=torch.bfloat16, device="cuda")
    ops.flip(wd, wt, cin, cout)
    dx = torch.empty(SHAPE + (cin,), dtype=torch.bfloat16, device="cuda")
    ops.conv(_dev(dy, ops), wt, None, dx, SHAPE, cout, cin, False)
    assert rel_l2(_host(dx, ops), dx_ref) <= 5e-3


def test_pool_upsample_concat_and_backward(ops):
    import torch

    rng = np.random.default_rng(5)
    shape = (2, 4, 6, 16)
    a = U.to_bf16(rng.standard_normal(shape + (16,)))
    p = torch.empty((2, 2, 3, 8, 16), dtype=torch.bfloat16, device="cuda")
    ops.pool(_dev(a, ops), p, shape, 16)
    assert rel_l2(_host(p, ops), U.pool(a)) <= 3e-3
    low = U.to_bf16(rng.standard_normal((2, 2, 3, 8, 32)))
    cat = torch.empty(shape + (48,), dtype=torch.bfloat16, device="cuda")
    ops.up_cat(_dev(low, ops), _dev(a, ops), cat, shape, 32, 16)
    assert np.array_equal(_host(cat, ops), np.concatenate([U.up(low), a], axis=-1))
    dcat = U.to_bf16(rng.standard_normal(shape + (48,)))
    dlow = torch.empty((2, 2, 3, 8, 32), dtype=torch.bfloat16, device="cuda")
    dskip = torch.empty(shape + (16,), dtype=torch.bfloat16, device="cuda")
    ops.up_cat_bwd(_dev(dcat, ops), dlow, dskip, shape, 32, 16)
    assert rel_l2(_host(dlow, ops), U.up_bwd(dcat[..., :32])) <= 3e-3
    assert np.array_equal(_host(dskip, ops), dcat[..., 32:])
    dp = U.to_bf16(rng.standard_normal((2, 2, 3, 8, 16)))
    ops.pool_bwd(_dev(dp, ops), dskip, shape, 16, True)  # += onto the skip gradient
    assert rel_l2(_host(dskip, ops), dcat[..., 32:] + U.pool_bwd(dp)) <= 3e-3


def _net_case(seed=0, shape=(1, 8, 8, 64)):
    rng = np.random.default_rng(seed)
    params = N.init_params(16, seed)
    for k in params:
        if k.endswith(".b"):
            params[k] = (0.05 * rng.standard_normal(params[k].shape)).astype(np.float32)
    x = np.zeros(shape + (16,), np.float32)
    x[..., :3] = rng.standard_normal(shape + (3,))
    target = rng.standard_normal(shape + (4,)).astype(np.float32)
    mask = (rng.random(shape) > 0.25).astype(np.uint8)
    cw = np.array([1.0, 1.0, 0.5, 0.5], np.float32)
    return params, x, target, mask, cw


def test_network_forward_backward_vs_oracle(engine):
    import torch

    params, x, target, mask, cw = _net_case()
    net = N.UNet3D(16, params=params)
    ops = net.ops
    count = float(mask.sum())
    out = net.forward(_dev(x, ops))
    loss = net.loss_and_grad(_dev(target, ops, False), torch.from_numpy(mask).cuda(), _dev(cw, ops, False), count)
    net.zero_grad()
    net.backward(net.D["out"])
    ref = U.UNetRef(params, bf16=True)
    ref_out = ref.forward(x)
    ref_loss, g = ref.loss(target.astype(np.float64), mask, cw.astype(np.float64), count)
    grads = ref.backward(g)
    assert rel_l2(_host(out, ops), ref_out) <= 2e-2
    assert abs(float(loss.item()) - ref_loss) <= 2e-2 * abs(ref_loss)
    for k in grads:
        got = _host(net.G[k], ops)
        assert rel_l2(got, grads[k]) <= 6e-2, (k, rel_l2(got, grads[k]))


def test_training_reduces_loss(gpu):
    import torch

    params, x, target, mask, cw = _net_case(seed=1)
    target = np.tanh(x[..., :4] * 0.7).astype(np.float32)  # a learnable map of the inputs
    net = N.UNet3D(16, params=params)
    ops = net.ops
    xd, td, md, cd = _dev(x, ops), _dev(target, ops, False), torch.from_numpy(mask).cuda(), _dev(cw, ops, False)
    losses = []
    for _ in range(60):
        net.forward(xd)
        loss = net.loss_and_grad(td, md, cd, float(mask.sum()))
        net.zero_grad()
        net.backward(net.D["out"])
        net.adam_step(lr=3e-3)
        losses.append(float(loss.item()))
    assert np.isfinite(losses).all()
    assert losses[-1] < 0.6 * losses[0], losses[::10]
    assert losses[-1] < min(losses[:10])


def test_features_on_gpu_match_host(gpu):
    import torch

    from lbm3d_bb_b200 import warmstart as W

    ops = N.Ops()
    for seed in (0, 7, 100003):
        p = W.case_params(seed)
        f = W.features(p)
        out = torch.empty((W.NZ, W.NY, W.NX, 16), dtype=torch.bfloat16, device="cuda")
        W.features_device(p, out, ops)
        g = _host(out, ops)
        assert np.array_equal(g[..., 0], f[..., 0])  # the solver's mask, bit for bit
        assert np.abs(g[..., 1:] - U.to_bf16(f[..., 1:])).max() <= 2 ** -7 * 4
        # and the solver rasterises the same solid nodes
        d = W.make_domain(p)
        assert np.array_equal(d.flags()[0].reshape(W.NZ, W.NY, W.NX), f[..., 0].astype(np.uint8))
        d.close()


@pytest.mark.parametrize("fy,fz", [(False, False), (True, False), (False, True), (True, True)])
def test_unpack_fields_undoes_mirroring(ops, fy, fz):
    import torch

    rng = np.random.default_rng(2)
    shape = (2, 4, 6, 16)
    y = U.to_bf16(rng.standard_normal(shape + (16,)))
    acc = torch.full((2, 4) + shape[1:], 7.0, dtype=torch.float32, device="cuda")
    ops.unpack_fields(_dev(y, ops), acc, shape, fy, fz, 0.5, False)
    ref = y[..., :4].copy()
    if fy:
        ref = ref[:, :, ::-1]
        ref[..., 2] *= -1
    if fz:
        ref = ref[:, ::-1]
        ref[..., 3] *= -1
    ref = 0.5 * np.moveaxis(ref, -1, 1)
    assert np.array_equal(_host(acc, ops), ref)
    ops.unpack_fields(_dev(y, ops), acc, shape, fy, fz, 0.5, True)
    assert np.array_equal(_host(acc, ops), 2 * ref)
