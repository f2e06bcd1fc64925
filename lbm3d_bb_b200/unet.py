"""3-D U-Net of the learned warm start, driven through libunet3d.so (include/unet3d.h).

Three levels, base width w (16): two 3x3x3 convolutions with ReLU per level on the
way down (2x2x2 average pooling between levels), nearest upsampling and skip
concatenation on the way up, and a 3x3x3 head.  Inputs: 16 channels (the features
of ``features()`` padded with zeros); outputs: 16 channels of which the first four
are the normalised steady fields (rho - 1) / (3 u^2), u_x / u, u_y / u, u_z / u.

Every operation is a kernel of libunet3d.so; torch tensors only hold the device
memory.  Master weights, gradients and Adam moments are FP32, the working weights
and activations BF16 (tensor-core MMA with FP32 accumulation).
"""
from __future__ import annotations

import ctypes as C
import math
import os
from pathlib import Path
from typing import Optional

import numpy as np

IN_CH = 16   # padded input channels
OUT_CH = 16  # padded output channels
N_TARGET = 4

_lib = None
LIB_PATH = Path(os.environ.get("UNET3D_LIB", Path(__file__).resolve().parent / "libunet3d.so"))


class NnError(RuntimeError):
    pass


def lib() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(f"{LIB_PATH} is missing (build it with `python -m lbm3d_bb_b200.build`)")
    L = C.CDLL(str(LIB_PATH))
    vp, i32, i64, f32, f64 = C.c_void_p, C.c_int32, C.c_int64, C.c_float, C.c_double
    proto = {
        "nn_abi_version": (i32, []),
        "nn_last_error": (C.c_char_p, []),
        "nn_conv3d_fwd": (i32, [vp, vp, vp, vp, i32, i32, i32, i32, i32, i32, i32, vp]),
        "nn_conv3d_flip": (i32, [vp, vp, i32, i32, vp]),
        "nn_conv3d_bwd_weight": (i32, [vp, vp, vp, i32, i32, i32, i32, i32, i32, vp]),
        "nn_bias_grad": (i32, [vp, vp, i64, i32, vp]),
        "nn_relu_bwd": (i32, [vp, vp, i64, vp]),
        "nn_pool2": (i32, [vp, vp, i32, i32, i32, i32, i32, vp]),
        "nn_pool2_bwd": (i32, [vp, vp, i32, i32, i32, i32, i32, i32, vp]),
        "nn_up2_concat": (i32, [vp, vp, vp, i32, i32, i32, i32, i32, i32, vp]),
        "nn_up2_concat_bwd": (i32, [vp, vp, vp, i32, i32, i32, i32, i32, i32, vp]),
        "nn_mse": (i32, [vp, vp, vp, vp, vp, vp, i64, i32, i32, f64, vp]),
        "nn_adam": (i32, [vp, vp, vp, vp, vp, i64, f32, f32, f32, f32, i32, vp]),
        "nn_diff_norms": (i32, [vp, vp, i64, vp, vp]),
        "nn_features_ellipsoid": (i32, [vp, i32, i32, i32, vp, vp, vp, f32, vp]),
        "nn_unpack_fields": (i32, [vp, vp, i32, i32, i32, i32, i32, i32, f32, i32, vp]),
        "nn_set_conv_engine": (i32, [i32]),
        "nn_conv_uses_tma": (i32, [i32, i32, i32, i32]),
        "nn_tc_status": (i32, [vp]),
        "nn_wait_selftest": (i32, [i32, vp]),
        "nn_to_bf16": (i32, [vp, vp, i64, vp]),
        "nn_from_bf16": (i32, [vp, vp, i64, vp]),
    }
    for name, (res, args) in proto.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def exported_symbols() -> list[str]:
    return ["nn_abi_version", "nn_last_error", "nn_set_conv_engine", "nn_conv_uses_tma", "nn_tc_status", "nn_wait_selftest", "nn_conv3d_fwd", "nn_conv3d_flip", "nn_conv3d_bwd_weight",
            "nn_bias_grad", "nn_relu_bwd", "nn_pool2", "nn_pool2_bwd", "nn_up2_concat", "nn_up2_concat_bwd",
            "nn_mse", "nn_adam", "nn_diff_norms", "nn_features_ellipsoid", "nn_unpack_fields", "nn_to_bf16",
            "nn_from_bf16"]


ENGINES = {"mma": 0, "tcgen05": 1, "auto": 2, "tcgen05-tma": 3}


def set_conv_engine(name: str) -> str:
    """Selects the forward-convolution kernels ('mma', 'tcgen05', 'auto': tcgen05 for
    Cout >= 32, or 'tcgen05-tma'); returns the previous one."""
    prev = lib().nn_set_conv_engine(ENGINES[name])
    if prev not in (0, 1, 2, 3):
        raise NnError((lib().nn_last_error() or b"").decode(errors="replace"))
    return {v: k for k, v in ENGINES.items()}[prev]


def tc_status(stream=None) -> None:
    """Raises NnError when a tcgen05 convolution gave up waiting since the last check."""
    _ck(lib().nn_tc_status(C.c_void_p(getattr(stream, "cuda_stream", stream) or 0)))


def _ck(status: int) -> None:
    if status != 0:
        raise NnError((lib().nn_last_error() or b"").decode(errors="replace"))


def _p(t) -> Optional[int]:
    return None if t is None else int(t.data_ptr())


class Ops:
    """Thin typed calls of libunet3d.so on one stream (torch tensors in, nothing returned)."""

    def __init__(self, stream=None):
        self.L = lib()
        self.s = C.c_void_p(getattr(stream, "cuda_stream", stream) or 0)

    def conv(self, x, w, b, y, shape, cin, cout, relu):
        n, d, h, wd = shape
        _ck(self.L.nn_conv3d_fwd(_p(x), _p(w), _p(b), _p(y), n, d, h, wd, cin, cout, int(relu), self.s))

    def flip(self, w, wt, cin, cout):
        _ck(self.L.nn_conv3d_flip(_p(w), _p(wt), cin, cout, self.s))

    def bwd_weight(self, x, dy, dw, shape, cin, cout):
        n, d, h, wd = shape
        _ck(self.L.nn_conv3d_bwd_weight(_p(x), _p(dy), _p(dw), n, d, h, wd, cin, cout, self.s))

    def bias_grad(self, dy, db, voxels, c):
        _ck(self.L.nn_bias_grad(_p(dy), _p(db), voxels, c, self.s))

    def relu_bwd(self, dy, y):
        _ck(self.L.nn_relu_bwd(_p(dy), _p(y), dy.numel(), self.s))

    def pool(self, x, y, shape, c):
        _ck(self.L.nn_pool2(_p(x), _p(y), *shape, c, self.s))

    def pool_bwd(self, dy, dx, shape, c, accumulate):
        _ck(self.L.nn_pool2_bwd(_p(dy), _p(dx), *shape, c, int(accumulate), self.s))

    def up_cat(self, low, skip, y, shape, cu, cs):
        _ck(self.L.nn_up2_concat(_p(low), _p(skip), _p(y), *shape, cu, cs, self.s))

    def up_cat_bwd(self, dcat, dlow, dskip, shape, cu, cs):
        _ck(self.L.nn_up2_concat_bwd(_p(dcat), _p(dlow), _p(dskip), *shape, cu, cs, self.s))

    def mse(self, out, target, mask, cw, dout, loss, voxels, count):
        _ck(self.L.nn_mse(_p(out), _p(target), _p(mask), _p(cw), _p(dout), _p(loss), voxels, OUT_CH, N_TARGET,
                          float(count), self.s))

    def adam(self, w, g, m, v, wb, lr, b1, b2, eps, t):
        _ck(self.L.nn_adam(_p(w), _p(g), _p(m), _p(v), _p(wb), w.numel(), lr, b1, b2, eps, t, self.s))

    def diff_norms(self, a, b, out):
        _ck(self.L.nn_diff_norms(_p(a), _p(b), a.numel(), _p(out), self.s))

    def features_ellipsoid(self, out, shape_xyz, center, rot, semi, re_feature):
        c = (C.c_double * 3)(*center)
        r = (C.c_double * 9)(*rot)
        s = (C.c_double * 3)(*semi)
        nx, ny, nz = shape_xyz
        _ck(self.L.nn_features_ellipsoid(_p(out), nx, ny, nz, c, r, s, float(re_feature), self.s))

    def unpack_fields(self, y, out, shape, flip_y, flip_z, weight, accumulate):
        n, d, h, wd = shape
        _ck(self.L.nn_unpack_fields(_p(y), _p(out), n, d, h, wd, int(flip_y), int(flip_z), float(weight),
                                    int(accumulate), self.s))

    def to_bf16(self, x, y):
        _ck(self.L.nn_to_bf16(_p(x), _p(y), x.numel(), self.s))

    def from_bf16(self, x, y):
        _ck(self.L.nn_from_bf16(_p(x), _p(y), x.numel(), self.s))


def layer_table(width: int = 16):
    """(name, cin, cout, relu) of the eleven convolutions, in forward order."""
    w = width
    return [("e1a", IN_CH, w, True), ("e1b", w, w, True),
            ("e2a", w, 2 * w, True), ("e2b", 2 * w, 2 * w, True),
            ("e3a", 2 * w, 4 * w, True), ("e3b", 4 * w, 4 * w, True),
            ("d2a", 6 * w, 2 * w, True), ("d2b", 2 * w, 2 * w, True),
            ("d1a", 3 * w, w, True), ("d1b", w, w, True),
            ("head", w, OUT_CH, False)]


def init_params(width: int = 16, seed: int = 0, n_inputs: int = 6) -> dict[str, np.ndarray]:
    """He-normal weights [27][cout][cin] (the padded input/output channels zero), zero
    biases; FP32 numpy arrays keyed '<layer>.w' / '<layer>.b'."""
    rng = np.random.default_rng(seed)
    params = {}
    for name, cin, cout, relu in layer_table(width):
        fan_in = 27 * (n_inputs if name == "e1a" else cin)
        std = math.sqrt((2.0 if relu else 1.0) / fan_in)
        w = (rng.standard_normal((27, cout, cin)) * std).astype(np.float32)
        if name == "e1a":
            w[:, :, n_inputs:] = 0.0
        if name == "head":
            w[:, N_TARGET:, :] = 0.0
        params[f"{name}.w"] = w
        params[f"{name}.b"] = np.zeros(cout, np.float32)
    return params


class UNet3D:
    """Parameters on one GPU plus the forward / backward passes for a batch shape."""

    def __init__(self, width: int = 16, device: int = 0, stream=None, params: Optional[dict] = None, seed: int = 0):
        import torch

        self.torch = torch
        self.width = width
        self.dev = torch.device(f"cuda:{device}")
        self.ops = Ops(stream)
        self.layers = layer_table(width)
        src = params if params is not None else init_params(width, seed)
        f32 = dict(dtype=torch.float32, device=self.dev)
        self.W = {k: torch.from_numpy(np.ascontiguousarray(v, np.float32)).to(**f32) for k, v in src.items()}
        self.Wb = {}
        for name, cin, cout, _ in self.layers:
            self.Wb[name] = torch.empty((27, cout, cin), dtype=torch.bfloat16, device=self.dev)
            self.ops.to_bf16(self.W[f"{name}.w"], self.Wb[name])
        self.G = {k: torch.zeros_like(v) for k, v in self.W.items()}
        self.M = {k: torch.zeros_like(v) for k, v in self.W.items()}
        self.V = {k: torch.zeros_like(v) for k, v in self.W.items()}
        self.t = 0
        self._shape = None

    # -- buffers -----------------------------------------------------------------------
    def _alloc(self, shape):
        if self._shape == shape:
            return
        t = self.torch
        n, d, h, wd = shape
        w = self.width
        L1, L2, L3 = (n, d, h, wd), (n, d // 2, h // 2, wd // 2), (n, d // 4, h // 4, wd // 4)
        self.geo = {1: L1, 2: L2, 3: L3}
        chans = {"x": (1, IN_CH), "a1": (1, w), "s1": (1, w), "p1": (2, w), "a2": (2, 2 * w), "s2": (2, 2 * w),
                 "p2": (3, 2 * w), "a3": (3, 4 * w), "b3": (3, 4 * w), "c2": (2, 6 * w), "a4": (2, 2 * w),
                 "a5": (2, 2 * w), "c1": (1, 3 * w), "a6": (1, w), "a7": (1, w), "out": (1, OUT_CH)}
        bf = dict(dtype=t.bfloat16, device=self.dev)
        self.A = {k: t.empty((*self.geo[lv], c), **bf) for k, (lv, c) in chans.items()}
        self.D = {k: t.empty((*self.geo[lv], c), **bf) for k, (lv, c) in chans.items() if k != "x"}
        self.Wt = {name: t.empty((27, cin, cout), **bf) for name, cin, cout, _ in self.layers}
        self._shape = shape

    # -- passes ------------------------------------------------------------------------
    def _conv(self, name, x, y, lv):
        cin, cout, relu = next((ci, co, r) for nm, ci, co, r in self.layers if nm == name)
        self.ops.conv(x, self.Wb[name], self.W[f"{name}.b"], y, self.geo[lv], cin, cout, relu)

    def forward(self, x):
        """x: BF16 (n, d, h, w, 16) with w % 64 == 0 and d, h % 4 == 0; returns the
        BF16 output buffer (n, d, h, w, 16), valid until the next call."""
        shape = tuple(int(s) for s in x.shape[:4])
        self._alloc(shape)
        A, o, w = self.A, self.ops, self.width
        A["x"].copy_(x)
        self._conv("e1a", A["x"], A["a1"], 1)
        self._conv("e1b", A["a1"], A["s1"], 1)
        o.pool(A["s1"], A["p1"], self.geo[1], w)
        self._conv("e2a", A["p1"], A["a2"], 2)
        self._conv("e2b", A["a2"], A["s2"], 2)
        o.pool(A["s2"], A["p2"], self.geo[2], 2 * w)
        self._conv("e3a", A["p2"], A["a3"], 3)
        self._conv("e3b", A["a3"], A["b3"], 3)
        o.up_cat(A["b3"], A["s2"], A["c2"], self.geo[2], 4 * w, 2 * w)
        self._conv("d2a", A["c2"], A["a4"], 2)
        self._conv("d2b", A["a4"], A["a5"], 2)
        o.up_cat(A["a5"], A["s1"], A["c1"], self.geo[1], 2 * w, w)
        self._conv("d1a", A["c1"], A["a6"], 1)
        self._conv("d1b", A["a6"], A["a7"], 1)
        self._conv("head", A["a7"], A["out"], 1)
        return A["out"]

    def _back(self, name, x, g, dx, lv, y=None):
        """g: gradient at the layer output (masked through ReLU with y when given);
        accumulates the parameter gradients and writes the input gradient to dx."""
        cin, cout, relu = next((ci, co, r) for nm, ci, co, r in self.layers if nm == name)
        if relu:
            self.ops.relu_bwd(g, y)
        geo = self.geo[lv]
        vox = geo[0] * geo[1] * geo[2] * geo[3]
        self.ops.bwd_weight(x, g, self.G[f"{name}.w"], geo, cin, cout)
        self.ops.bias_grad(g, self.G[f"{name}.b"], vox, cout)
        if dx is not None:
            self.ops.flip(self.Wb[name], self.Wt[name], cin, cout)
            self.ops.conv(g, self.Wt[name], None, dx, geo, cout, cin, False)

    def backward(self, dout):
        """dout: gradient of the loss at the output (BF16, like forward's result).
        Adds into the FP32 gradients (zero them with zero_grad)."""
        A, D, o, w = self.A, self.D, self.ops, self.width
        D["out"].copy_(dout) if dout.data_ptr() != D["out"].data_ptr() else None
        self._back("head", A["a7"], D["out"], D["a7"], 1)
        self._back("d1b", A["a6"], D["a7"], D["a6"], 1, A["a7"])
        self._back("d1a", A["c1"], D["a6"], D["c1"], 1, A["a6"])
        o.up_cat_bwd(D["c1"], D["a5"], D["s1"], self.geo[1], 2 * w, w)
        self._back("d2b", A["a4"], D["a5"], D["a4"], 2, A["a5"])
        self._back("d2a", A["c2"], D["a4"], D["c2"], 2, A["a4"])
        o.up_cat_bwd(D["c2"], D["b3"], D["s2"], self.geo[2], 4 * w, 2 * w)
        self._back("e3b", A["a3"], D["b3"], D["a3"], 3, A["b3"])
        self._back("e3a", A["p2"], D["a3"], D["p2"], 3, A["a3"])
        o.pool_bwd(D["p2"], D["s2"], self.geo[2], 2 * w, True)
        self._back("e2b", A["a2"], D["s2"], D["a2"], 2, A["s2"])
        self._back("e2a", A["p1"], D["a2"], D["p1"], 2, A["a2"])
        o.pool_bwd(D["p1"], D["s1"], self.geo[1], w, True)
        self._back("e1b", A["a1"], D["s1"], D["a1"], 1, A["s1"])
        self._back("e1a", A["x"], D["a1"], None, 1, A["a1"])

    def zero_grad(self):
        for g in self.G.values():
            g.zero_()

    def loss_and_grad(self, target, mask, cw, count, accumulate=None):
        """Masked MSE of the last forward output; writes its gradient into the output
        gradient buffer and returns the loss as a device FP64 scalar (added into
        `accumulate` when given)."""
        t = self.torch
        loss = accumulate if accumulate is not None else t.zeros(1, dtype=t.float64, device=self.dev)
        geo = self.geo[1]
        vox = geo[0] * geo[1] * geo[2] * geo[3]
        self.ops.mse(self.A["out"], target, mask, cw, self.D["out"], loss, vox, count)
        return loss

    def adam_step(self, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
        self.t += 1
        for name, cin, cout, _ in self.layers:
            self.ops.adam(self.W[f"{name}.w"], self.G[f"{name}.w"], self.M[f"{name}.w"], self.V[f"{name}.w"],
                          self.Wb[name], lr, b1, b2, eps, self.t)
            self.ops.adam(self.W[f"{name}.b"], self.G[f"{name}.b"], self.M[f"{name}.b"], self.V[f"{name}.b"], None,
                          lr, b1, b2, eps, self.t)
        # the zero-padded channels stay zero (their gradients are zero up to the
        # input/output padding, which carries no signal)

    def params_numpy(self) -> dict[str, np.ndarray]:
        return {k: v.detach().cpu().numpy() for k, v in self.W.items()}

    def save(self, path) -> None:
        np.savez(path, width=self.width, **self.params_numpy())

    @classmethod
    def load(cls, path, device: int = 0, stream=None) -> "UNet3D":
        z = np.load(path)
        params = {k: z[k] for k in z.files if k != "width"}
        return cls(int(z["width"]), device, stream, params)


def _conv_cli(argv=None) -> None:
    """Times repeated launches of one convolution layer (zero tensors):
    python -m lbm3d_bb_b200.unet --engine tcgen05 --shape 2,64,64,128 --cin 48 --cout 16 --launches 4"""
    import argparse

    import torch

    ap = argparse.ArgumentParser()
    ap.add_argument("--engine", default="auto", choices=sorted(ENGINES))
    ap.add_argument("--shape", default="2,64,64,128", help="n,d,h,w")
    ap.add_argument("--cin", type=int, default=48)
    ap.add_argument("--cout", type=int, default=16)
    ap.add_argument("--launches", type=int, default=4)
    args = ap.parse_args(argv)
    n, d, h, w = (int(v) for v in args.shape.split(","))
    set_conv_engine(args.engine)
    ops = Ops()
    x = torch.zeros((n, d, h, w, args.cin), dtype=torch.bfloat16, device="cuda")
    y = torch.empty((n, d, h, w, args.cout), dtype=torch.bfloat16, device="cuda")
    wt = torch.zeros((27, args.cout, args.cin), dtype=torch.bfloat16, device="cuda")
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.launches):
        ops.conv(x, wt, None, y, (n, d, h, w), args.cin, args.cout, True)
    e1.record()
    e1.synchronize()
    tc_status()
    ms = e0.elapsed_time(e1) / args.launches
    flops = 2.0 * n * d * h * w * 27 * args.cin * args.cout
    print(f"{args.engine}: {ms:.3f} ms per launch, {flops / (ms * 1e-3) / 1e12:.1f} TFLOP/s")


if __name__ == "__main__":
    _conv_cli()
