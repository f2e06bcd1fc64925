"""Pins the CPU restatement of the warm-start U-Net (oracle/unet_ref.py): its
analytic gradients against central finite differences of its own FP64 loss."""
import zlib

import numpy as np
import pytest

from lbm3d_bb_b200.unet import init_params
from oracle import unet_ref as U


def _setup(seed=0):
    rng = np.random.default_rng(seed)
    params = {k: v.astype(np.float64) for k, v in init_params(16, seed).items()}
    for k in params:
        if k.endswith(".b"):
            params[k] = 0.05 * rng.standard_normal(params[k].shape)
    shape = (1, 4, 4, 8)
    x = np.zeros(shape + (16,))
    x[..., :3] = rng.standard_normal(shape + (3,))
    t = rng.standard_normal(shape + (4,))
    mask = (rng.random(shape) > 0.2).astype(np.uint8)
    cw = np.array([1.0, 1.0, 0.5, 0.5])
    return params, x, t, mask, cw


def _loss(net, x, t, mask, cw):
    net.forward(x)
    return net.loss(t, mask, cw, float(mask.sum()))


def test_bf16_rounding_is_nearest_even():
    # BF16 keeps 8 significant bits (spacing 2^-7 above 1): ties go to the even neighbour
    assert U.to_bf16(np.array([1.0 + 2 ** -8]))[0] == 1.0
    assert U.to_bf16(np.array([1.0 + 3 * 2 ** -8]))[0] == 1.0 + 2 ** -6
    assert U.to_bf16(np.array([1.0 + 2 ** -8 + 2 ** -12]))[0] == 1.0 + 2 ** -7
    assert U.to_bf16(np.array([-2.5]))[0] == -2.5
    assert abs(U.to_bf16(np.array([3.0e-3]))[0] - 3.0e-3) / 3.0e-3 < 2 ** -8


def test_conv_adjoint_identity():
    """<conv(x), y> == <x, conv_bwd(y).dx> and <dw, w'> matches the directional
    derivative: the shift conventions of the forward and backward agree."""
    rng = np.random.default_rng(1)
    x = rng.standard_normal((2, 3, 4, 5, 16))
    w = rng.standard_normal((27, 8, 16))
    y = rng.standard_normal((2, 3, 4, 5, 8))
    dx, dw, db = U.conv_bwd(x, w, y)
    assert abs(np.sum(U.conv(x, w, None) * y) - np.sum(x * dx)) < 1e-9 * abs(np.sum(x * dx))
    w2 = rng.standard_normal(w.shape)
    assert abs(np.sum(U.conv(x, w2, None) * y) - np.sum(dw * w2)) < 1e-9 * abs(np.sum(dw * w2))
    assert np.allclose(db, y.reshape(-1, 8).sum(0))


@pytest.mark.parametrize("layer", U.LAYERS)
def test_gradients_match_finite_differences(layer):
    params, x, t, mask, cw = _setup()
    net = U.UNetRef(params, bf16=False)
    _, g = _loss(net, x, t, mask, cw)
    grads = net.backward(g)
    rng = np.random.default_rng(zlib.crc32(layer.encode()))
    for key in (f"{layer}.w", f"{layer}.b"):
        p = params[key]
        flat = np.flatnonzero(np.abs(grads[key]).ravel() > 1e-6 * np.abs(grads[key]).max())
        for idx in rng.choice(flat, size=min(4, flat.size), replace=False):
            eps = 1e-6
            vals = []
            for s in (+1, -1):
                q = {k: v.copy() for k, v in params.items()}
                q[key].ravel()[idx] = p.ravel()[idx] + s * eps
                vals.append(_loss(U.UNetRef(q, bf16=False), x, t, mask, cw)[0])
            fd = (vals[0] - vals[1]) / (2 * eps)
            an = grads[key].ravel()[idx]
            assert abs(fd - an) <= 1e-4 * abs(an) + 1e-10, (key, idx, fd, an)
