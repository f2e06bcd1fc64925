"""Learned warm start: steady channel flows past a random ellipsoid, generated by the
batched LBM, a 3-D U-Net trained on them with the project's own kernels
(libunet3d.so), and runs started from its prediction against runs started from rest.

Workload (one case per seed, numpy default_rng(seed)): a 128 x 64 x 64 D3Q19 BGK
channel, FP32 populations, equilibrium inlet u_x = 0.05 at x = 0, pressure outlet at
x = 127, no-slip walls on the y/z faces; one ellipsoid with semi-axes U[4, 12], a
uniformly random orientation (unit quaternion from four normal deviates) and centre
x in [24, 48], y and z in the central third; Re uniform in [10, 100] on the length
L = 2 * (largest semi-axis), tau = 1/2 + 3 u L / Re.

Network inputs (16 channels, 6 used): solid mask, approximate signed distance to the
ellipsoid / 16 (clipped to [-1, 4]), (Re - 55) / 45, and the node position x/NX, y/NY,
z/NZ (without it the network cannot place the developing channel profile along x, which
lies beyond its receptive field).  Outputs: (rho - 1) / (3 u^2), u_x / u, u_y / u,
u_z / u, trained with a masked MSE over the fluid nodes (Adam, cosine learning-rate decay).

A run is steady when the relative change of the field ||u(t) - u(t-100)|| / ||u(t)||
falls below `tol` (data generation), and its drag is steady when the relative drag
change over 100 steps stays below `drag_tol` for three checks in a row (evaluation).
A warm start computes the first-step residual ||u(1) - u(0)|| / ||u(0)||; above
`fallback` the case restarts from rest (the plain method remains the fallback).

Usage (one GPU):  python -m lbm3d_bb_b200.warmstart --train 2048 --heldout 256 --epochs 200 --group 128 \
                      [--time-budget SECONDS] --out DIR
                  python -m lbm3d_bb_b200.warmstart --heldout 256 --eval-weights WEIGHTS.npz --out DIR
"""
from __future__ import annotations

import argparse
import json
import math
import time
from pathlib import Path
from typing import Sequence

import numpy as np

from . import abi

NX, NY, NZ = 128, 64, 64
U_IN = 0.05
RHO_SCALE = 3.0 * U_IN * U_IN
CHANNEL = ("inlet", "pressure", "wall", "wall", "wall", "wall")
CHANNEL_WEIGHTS = (1.0, 1.0, 1.0, 1.0)


def quat_rotation(q) -> np.ndarray:
    """Row-major body->world rotation of a (not necessarily unit) quaternion."""
    w, x, y, z = np.asarray(q, np.float64) / np.linalg.norm(q)
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)],
                     [2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)],
                     [2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)]])


def case_params(seed: int) -> dict:
    rng = np.random.default_rng(seed)
    semi = rng.uniform(4.0, 12.0, 3)
    rot = quat_rotation(rng.standard_normal(4))
    center = (rng.uniform(24.0, 48.0), rng.uniform(NY / 3, 2 * NY / 3), rng.uniform(NZ / 3, 2 * NZ / 3))
    re = rng.uniform(10.0, 100.0)
    L = 2.0 * semi.max()
    return {"seed": int(seed), "semi": semi.tolist(), "rot": rot.ravel().tolist(), "center": [float(c) for c in center],
            "Re": float(re), "tau": 0.5 + 3.0 * U_IN * L / re}


def make_domain(p: dict, storage: str = "fp32", device: int = 0, stream=None, history: int = 256):
    from .domain import Domain

    d = Domain(NX, NY, NZ, collision="BGK", storage=storage, faces=CHANNEL, omega_p=1.0 / p["tau"],
               face_u=[(U_IN, 0.0, 0.0)] + [(0.0, 0.0, 0.0)] * 5, compute_force=True, force_history=history,
               device=device, stream=stream)
    d.add_body(abi.make_body(abi.BODY_ELLIPSOID, p["center"], semi=p["semi"], rot=p["rot"]))
    return d


N_FEATURES = 6
_GRID = None


def _grid():
    global _GRID
    if _GRID is None:
        _GRID = np.meshgrid(np.arange(NZ) + 0.5, np.arange(NY) + 0.5, np.arange(NX) + 0.5, indexing="ij")
    return _GRID


def features(p: dict) -> np.ndarray:
    """(NZ, NY, NX, 16) float32 network input of a case."""
    z, y, x = _grid()
    r = np.asarray(p["rot"]).reshape(3, 3)
    dx, dy, dz = x - p["center"][0], y - p["center"][1], z - p["center"][2]
    b = [(r[0, k] * dx + r[1, k] * dy) + r[2, k] * dz for k in range(3)]
    s = p["semi"]
    q = [b[k] / s[k] for k in range(3)]
    e2 = (q[0] * q[0] + q[1] * q[1]) + q[2] * q[2]  # same expression as the rasteriser
    e = np.sqrt(e2)
    grad = np.sqrt(sum((b[k] / (s[k] * s[k])) ** 2 for k in range(3))) / np.maximum(e, 1e-12)
    sdf = (e - 1.0) / np.maximum(grad, 1e-12)  # first-order distance to the surface
    f = np.zeros((NZ, NY, NX, 16), np.float32)
    f[..., 0] = e2 <= 1.0
    f[..., 1] = np.clip(sdf / 16.0, -1.0, 4.0)
    f[..., 2] = (p["Re"] - 55.0) / 45.0
    f[..., 3] = x / NX
    f[..., 4] = y / NY
    f[..., 5] = z / NZ
    return f


REFLECTIONS = ((False, False), (True, False), (False, True), (True, True))  # (mirror y, mirror z)


def reflect(p: dict, flip_y: bool, flip_z: bool) -> dict:
    """The case mirrored about the channel's mid-plane(s): the ellipsoid's centre is
    mirrored and its rotation becomes F R F (F = the mirror), a proper rotation of the
    mirrored body; flow fields mirror with u_y (u_z) negated."""
    f = np.diag([1.0, -1.0 if flip_y else 1.0, -1.0 if flip_z else 1.0])
    r = np.asarray(p["rot"]).reshape(3, 3)
    c = list(p["center"])
    if flip_y:
        c[1] = NY - c[1]
    if flip_z:
        c[2] = NZ - c[2]
    q = dict(p)
    q["center"] = c
    q["rot"] = (f @ r @ f).ravel().tolist()
    return q


def mirror_target(t: np.ndarray, flip_y: bool, flip_z: bool) -> np.ndarray:
    """Target (NZ, NY, NX, 4) of the mirrored case."""
    t = t[:, ::-1] if flip_y else t
    t = t[::-1] if flip_z else t
    t = np.array(t)
    if flip_y:
        t[..., 2] = -t[..., 2]
    if flip_z:
        t[..., 3] = -t[..., 3]
    return t


def features_device(p: dict, out, ops) -> None:
    """features(p) computed on the GPU into a BF16 (NZ, NY, NX, 16) tensor."""
    ops.features_ellipsoid(out, (NX, NY, NZ), p["center"], p["rot"], p["semi"], (p["Re"] - 55.0) / 45.0)


def target_of(rho, u, v, w) -> np.ndarray:
    t = np.stack([(rho - 1.0) / RHO_SCALE, u / U_IN, v / U_IN, w / U_IN], axis=-1)
    return t.reshape(NZ, NY, NX, 4).astype(np.float32)


class Stepper:
    """A set of cases stepped together (one persistent launch per step, graph replay
    of `check` steps) with field and drag convergence tracking."""

    def __init__(self, params: Sequence[dict], device: int, stream, init=None, check: int = 100):
        import torch

        from .batch import Batch
        from .unet import Ops

        self.torch = torch
        self.params = list(params)
        self.check = check
        self.stream = stream
        self.doms = [make_domain(p, device=device, stream=stream, history=2 * check + 8) for p in self.params]
        for k, d in enumerate(self.doms):
            if init is None or init[k] is None:
                d.init_equilibrium()
            else:
                d.init_equilibrium(*init[k])
        self.active = list(range(len(self.doms)))
        self.batch = Batch(self.doms)
        self.batch.capture(check)
        self.ops = Ops(stream)
        n = NX * NY * NZ
        f32 = dict(dtype=torch.float32, device=f"cuda:{device}")
        self.u = [[torch.zeros(n, **f32) for _ in range(3)] for _ in self.doms]
        self.u_prev = [[torch.zeros(n, **f32) for _ in range(3)] for _ in self.doms]
        self.norms = torch.zeros((len(self.doms), 2), dtype=torch.float64, device=f"cuda:{device}")
        self.steps = 0

    def export_u(self, into):
        for d, u in zip(self.doms, into):
            d.macros_into(None, u[0], u[1], u[2])

    def field_change(self) -> np.ndarray:
        """||u - u_prev|| / ||u|| per case since the previous call (inf at the first)."""
        self.u, self.u_prev = self.u_prev, self.u
        self.export_u(self.u)
        self.norms.zero_()
        for k in range(len(self.doms)):
            for c in range(3):
                self.ops.diff_norms(self.u[k][c], self.u_prev[k][c], self.norms[k])
        nrm = self.norms.cpu().numpy()
        return np.sqrt(nrm[:, 0] / np.maximum(nrm[:, 1], 1e-300))

    def advance(self):
        if self.batch is not None:
            self.batch.replay(1)
        self.steps += self.check

    def retire(self, done) -> None:
        """Stops stepping the cases with done[k] true (steady or diverged): the batch and
        its captured graph are rebuilt over the others, so the set's device time follows
        the steps each case needs rather than the slowest case."""
        from .batch import Batch

        keep = [k for k in self.active if not done[k]]
        if len(keep) == len(self.active):
            return
        self.batch.close()
        self.active, self.batch = keep, None
        if keep:
            self.batch = Batch([self.doms[k] for k in keep])
            self.batch.capture(self.check)

    def drags(self) -> np.ndarray:
        """Drag `check` steps ago and now, shape (cases, 2) (NaN before enough steps)."""
        out = np.full((len(self.doms), 2), np.nan)
        for k, d in enumerate(self.doms):
            n = d.step_count
            if n - self.check >= 1:
                out[k] = (d.force(n - self.check)[0], d.force(n)[0])
        return out

    def close(self):
        if self.batch is not None:
            self.batch.close()
        for d in self.doms:
            d.close()


def generate(seeds: Sequence[int], device: int = 0, stream=None, max_steps: int = 30000, tol: float = 1e-6,
             group: int = 64, log=print, augment: bool = False):
    """Steady states of the cases, kept on the GPU: BF16 features (n, NZ, NY, NX, 16),
    FP32 targets (n, NZ, NY, NX, 4), fluid masks, fluid counts, and the record of
    each run (steps, stability).  With `augment`, each steady state also enters in its
    three mirror images (y, z, both)."""
    import torch

    from .unet import Ops

    ops = Ops(stream)
    dev = torch.device(f"cuda:{device}")
    feats, targs, masks, counts, record = [], [], [], [], []
    for g0 in range(0, len(seeds), group):
        params = [case_params(s) for s in seeds[g0:g0 + group]]
        st = Stepper(params, device, stream)
        done = np.zeros(len(params), bool)
        steps = np.full(len(params), -1)
        st.field_change()
        t0 = time.perf_counter()
        while st.steps < max_steps and not done.all():
            st.advance()
            ch = st.field_change()
            newly = (~done) & (ch < tol)
            steps[newly] = st.steps
            done |= newly | ~np.isfinite(ch)
            st.retire(done)  # settled or diverged cases stop stepping
        torch.cuda.synchronize()
        log(f"group {g0 // group}: {len(params)} cases, {st.steps} steps, {time.perf_counter() - t0:.1f} s, "
            f"converged {(steps > 0).sum()}")
        for k, (p, d) in enumerate(zip(params, st.doms)):
            rho, u, v, w = d.macros(np.float32)
            ok = bool(np.isfinite(u).all() and np.isfinite(rho).all())
            record.append({"seed": p["seed"], "Re": p["Re"], "tau": p["tau"], "steps_to_steady": int(steps[k]),
                           "stable": ok})
            if not ok:
                continue
            t0_ = target_of(rho, u, v, w)
            m0 = (d.flags()[0] == 0).reshape(NZ, NY, NX).astype(np.uint8)
            for fy, fz in (REFLECTIONS if augment else REFLECTIONS[:1]):
                xb = torch.empty((NZ, NY, NX, 16), dtype=torch.bfloat16, device=dev)
                features_device(reflect(p, fy, fz), xb, ops)
                feats.append(xb)
                targs.append(torch.from_numpy(mirror_target(t0_, fy, fz)).to(dev))
                m = m0[:, ::-1] if fy else m0
                m = np.ascontiguousarray(m[::-1] if fz else m)
                masks.append(torch.from_numpy(m).to(dev))
                counts.append(int(m.sum()))
        st.close()
    return torch.stack(feats), torch.stack(targs), torch.stack(masks), np.array(counts), record


def epochs_within(seconds: float, step_s: float, n: int, batch: int, wanted: int) -> int:
    """Epochs of `n` samples in mini-batches of `batch` that fit `seconds` at `step_s` per
    training step: at least one, at most `wanted`."""
    per_epoch = step_s * max(1, n // batch)
    fit = int(seconds / per_epoch) if per_epoch > 0 else wanted
    return max(1, min(wanted, fit))


def train(model, X, T, M, counts, epochs: int, batch: int = 4, lr: float = 1e-3, seed: int = 0, log=print,
          lr_min: float = 1e-5, weights=CHANNEL_WEIGHTS):
    """Adam on the masked MSE over the GPU-resident data set (shuffled mini-batches
    gathered by index), learning rate decayed from lr to lr_min on a cosine.  Returns
    the per-epoch mean loss."""
    import torch

    dev = model.dev
    n = X.shape[0]
    cw = torch.tensor(weights, dtype=torch.float32, device=dev)
    acc = torch.zeros(1, dtype=torch.float64, device=dev)
    rng = np.random.default_rng(seed)
    hist = []
    nb = max(1, n // batch)
    total = max(1, epochs * nb)
    t = 0
    for ep in range(epochs):
        order = rng.permutation(n)
        acc.zero_()
        for b0 in range(0, nb * batch, batch):
            sel = order[b0:b0 + batch]
            idx = torch.from_numpy(sel).to(dev)
            model.forward(X.index_select(0, idx))
            model.loss_and_grad(T.index_select(0, idx), M.index_select(0, idx), cw, float(counts[sel].sum()),
                                accumulate=acc)
            model.zero_grad()
            model.backward(model.D["out"])
            model.adam_step(lr=lr_min + 0.5 * (lr - lr_min) * (1.0 + math.cos(math.pi * t / total)))
            t += 1
        hist.append(float(acc.item()) / nb)
        if ep % 10 == 0 or ep == epochs - 1:
            log(f"epoch {ep}: loss {hist[-1]:.5f}")
    return hist


def predict(model, params: Sequence[dict], mirror_average: bool = False):
    """Equilibrium initial fields (rho, u, v, w as FP64 host arrays) per case; with
    `mirror_average` the network sees the case in its four mirror images (one batch)
    and the predictions, mapped back, are averaged."""
    import torch

    out = []
    dev = model.dev
    refl = REFLECTIONS if mirror_average else REFLECTIONS[:1]
    xb = torch.empty((len(refl), NZ, NY, NX, 16), dtype=torch.bfloat16, device=dev)
    acc = torch.empty((1, 4, NZ, NY, NX), dtype=torch.float32, device=dev)
    for p in params:
        for k, (fy, fz) in enumerate(refl):
            features_device(reflect(p, fy, fz), xb[k], model.ops)
        y = model.forward(xb)
        for k, (fy, fz) in enumerate(refl):
            model.ops.unpack_fields(y[k:k + 1], acc, (1, NZ, NY, NX), fy, fz, 1.0 / len(refl), k > 0)
        o = acc.cpu().numpy().reshape(4, -1).astype(np.float64)
        out.append((1.0 + RHO_SCALE * o[0], U_IN * o[1], U_IN * o[2], U_IN * o[3]))
    return out


MIN_STEPS = int(NX / U_IN)  # one flow-through time: the drag is not checked earlier


def run_to_steady_drag(params, device, stream, init=None, drag_tol=1e-5, max_steps=40000, fallback=None):
    """Steps every case until its drag is steady; returns per-case steps (0: diverged,
    -1: not steady by max_steps), final drag, fallbacks, and the device time of the
    whole set (CUDA events, set-up included)."""
    import torch

    n = len(params)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    st = Stepper(params, device, stream, init=init)
    fell_back = np.zeros(n, bool)
    if fallback is not None and init is not None:
        # first-step residual of the prediction; too large -> restart from rest
        st.export_u(st.u)
        for d in st.doms:
            d.step(1)
        ch = st.field_change()
        fell_back = ~(ch <= fallback)
        for k in np.flatnonzero(fell_back):
            st.doms[k].init_equilibrium()
    calm = np.zeros(n, int)
    steps = np.full(n, -1)
    while (steps < 0).any() and max(st.doms[k].step_count for k in st.active) < max_steps:
        st.advance()
        dr = st.drags()
        rel = np.abs(dr[:, 1] - dr[:, 0]) / np.maximum(np.abs(dr[:, 1]), 1e-12)
        counts = np.array([d.step_count for d in st.doms])
        ok = np.isfinite(rel) & (rel < drag_tol) & (np.abs(dr[:, 1]) > 0) & (counts >= MIN_STEPS)
        calm = np.where(ok, calm + 1, 0)
        newly = (steps < 0) & (calm >= 3)
        steps[newly] = counts[newly]
        diverged = (steps < 0) & ~np.isfinite(dr[:, 1]) & (counts > st.check)
        steps[diverged] = 0
        st.retire(steps >= 0)
    e1.record(stream)
    e1.synchronize()
    drag = np.array([float(d.force()[0]) for d in st.doms])
    st.close()
    return {"steps": steps, "drag": drag, "fell_back": fell_back, "set_ms": e0.elapsed_time(e1)}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--train", type=int, default=256)
    ap.add_argument("--heldout", type=int, default=32)
    ap.add_argument("--epochs", type=int, default=200)
    ap.add_argument("--batch", type=int, default=4)
    ap.add_argument("--group", type=int, default=64, help="cases stepped together in data generation")
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--max-steps", type=int, default=40000, help="cap of the data-generation runs")
    ap.add_argument("--eval-max-steps", type=int, default=60000, help="cap of the evaluation runs")
    ap.add_argument("--tol", type=float, default=1e-5, help="field steadiness per 100 steps (FP32 rounding floor ~6e-7)")
    ap.add_argument("--drag-tol", type=float, default=1e-4, help="relative drag change per 100 steps, three checks in a row")
    ap.add_argument("--fallback", type=float, default=0.05)
    ap.add_argument("--rho-weight", type=float, default=1.0, help="loss weight of the density channel")
    ap.add_argument("--augment", action="store_true", help="train on the three mirror images of every state too")
    ap.add_argument("--mirror-average", action="store_true", help="average the prediction over the four mirror images")
    ap.add_argument("--time-budget", type=float, default=0.0,
                    help="wall seconds for the whole run: fewer epochs when training would not fit (0: no limit)")
    ap.add_argument("--eval-reserve", type=float, default=900.0, help="seconds kept for the evaluation under --time-budget")
    ap.add_argument("--out", default="warmstart_out")
    ap.add_argument("--eval-weights", default=None,
                    help="evaluate these saved weights on the held-out seeds (no data generation or training)")
    args = ap.parse_args(argv)
    import torch

    out = Path(args.out)
    out.mkdir(parents=True, exist_ok=True)
    logf = open(out / "log.txt", "a")

    def log(msg):
        print(msg, flush=True)
        logf.write(msg + "\n")
        logf.flush()

    torch.cuda.set_device(0)
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):  # torch's own copies and fills share the kernels' stream
        _run(args, stream, out, log)


def _run(args, stream, out, log):
    import torch

    from .unet import UNet3D

    t0 = time.perf_counter()
    train_seeds = list(range(args.train))
    held = list(range(100000, 100000 + args.heldout))
    if args.eval_weights:
        model = UNet3D.load(args.eval_weights, 0, stream)
        rec, hist, train_s, train_seeds = [], [float("nan")], 0.0, []
    else:
        X, T, M, counts, rec = generate(train_seeds, 0, stream, args.max_steps, args.tol, group=args.group, log=log,
                                        augment=args.augment)
        log(f"training set: {X.shape[0]} steady states of {len(train_seeds)} ({time.perf_counter() - t0:.0f} s)")
        epochs = args.epochs
        if args.time_budget > 0:
            # time a few training steps on a scratch network, then fit the epochs (and with
            # them the cosine schedule) into what is left of the budget
            probe = UNet3D(16, 0, stream, seed=1)
            train(probe, X[:8 * args.batch], T[:8 * args.batch], M[:8 * args.batch], counts[:8 * args.batch], 1,
                  args.batch, args.lr, log=lambda m: None)
            torch.cuda.synchronize()
            tp = time.perf_counter()
            train(probe, X[:8 * args.batch], T[:8 * args.batch], M[:8 * args.batch], counts[:8 * args.batch], 1,
                  args.batch, args.lr, log=lambda m: None)
            torch.cuda.synchronize()
            step_s = (time.perf_counter() - tp) / 8
            del probe
            left = args.time_budget - (time.perf_counter() - t0) - args.eval_reserve
            epochs = epochs_within(left, step_s, X.shape[0], args.batch, args.epochs)
            log(f"time budget: {step_s * 1e3:.1f} ms per training step, {left:.0f} s left for training: "
                f"{epochs} epochs")
        model = UNet3D(16, 0, stream, seed=0)
        t1 = time.perf_counter()
        hist = train(model, X, T, M, counts, epochs, args.batch, args.lr, log=log,
                     weights=(args.rho_weight,) + CHANNEL_WEIGHTS[1:])
        torch.cuda.synchronize()
        train_s = time.perf_counter() - t1
        model.save(out / "unet_c5.npz")
        del X, T, M
    params = [case_params(s) for s in held]
    # warm: inference (timed) + runs; rest: runs
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    init = predict(model, params, mirror_average=args.mirror_average)
    e1.record(stream)
    e1.synchronize()
    infer_ms = e0.elapsed_time(e1)
    warm = run_to_steady_drag(params, 0, stream, init=init, drag_tol=args.drag_tol, max_steps=args.eval_max_steps,
                              fallback=args.fallback)
    rest = run_to_steady_drag(params, 0, stream, init=None, drag_tol=args.drag_tol, max_steps=args.eval_max_steps)
    ok = (warm["steps"] > 0) & (rest["steps"] > 0)
    err = np.abs(warm["drag"] - rest["drag"]) / np.maximum(np.abs(rest["drag"]), 1e-30)
    res = {
        "train_cases": len(train_seeds), "train_steady": int(sum(r["stable"] and r["steps_to_steady"] > 0 for r in rec)),
        "epochs": len(hist) if not args.eval_weights else 0, "train_s": round(train_s, 1), "loss_first": hist[0], "loss_last": hist[-1],
        "heldout": len(held), "both_steady": int(ok.sum()),
        "rest_steps_mean": float(rest["steps"][ok].mean()) if ok.any() else None,
        "warm_steps_mean": float(warm["steps"][ok].mean()) if ok.any() else None,
        "step_ratio_mean": float(np.mean(rest["steps"][ok] / np.maximum(warm["steps"][ok], 1))) if ok.any() else None,
        "rest_set_ms": rest["set_ms"], "warm_set_ms": warm["set_ms"] + infer_ms, "inference_ms": infer_ms,
        "wall_speedup": rest["set_ms"] / (warm["set_ms"] + infer_ms),
        "drag_err_max": float(err[ok].max()) if ok.any() else None,
        "drag_err_median": float(np.median(err[ok])) if ok.any() else None,
        "fallbacks": int(warm["fell_back"].sum()),
        "per_case": [{"seed": s, "rest_steps": int(a), "warm_steps": int(b), "drag_rest": float(c),
                      "drag_warm": float(d), "fell_back": bool(f)}
                     for s, a, b, c, d, f in zip(held, rest["steps"], warm["steps"], rest["drag"], warm["drag"],
                                                 warm["fell_back"])],
        "data_record": rec, "loss_history": hist,
    }
    (out / "result.json").write_text(json.dumps(res, indent=1))
    log(json.dumps({k: v for k, v in res.items() if k not in ("per_case", "data_record", "loss_history")}))


if __name__ == "__main__":
    main()
