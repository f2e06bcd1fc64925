"""Accuracy of every storage form per workload, against FP64 (GPU) and the CPU oracle.

Run on a GPU box:  python -m tests.accuracy_report [--only c1,c2,c3,c4] [--out file.json]

  c1  sphere channel 96x48x48, BGK tau 0.8, 2000 steps: FP64 GPU vs FP64 oracle
      (fields and the per-step drag/lift history), FP32 / FP16-deviation drag vs FP64.
  c2  oscillating sphere 192x96x96, TRT tau+ 0.56, Lambda 3/16, 4000 steps: flags and
      links of the GPU bit-exact against the oracle after every body move of the first
      `oracle_steps` steps, populations of both in FP64; FP32 and FP16-deviation force
      histories against the FP64 GPU run over all steps.
  c3  porous periodic 512^3, BGK tau 0.6, g_x 1e-6, 1000 steps: mean u_x of FP32 and
      FP16-deviation against FP64.
  c4  the batched sweep (FP32, one persistent launch per step): per-domain drag against
      the same domains in FP64 on the GPU, and a subset against the FP64 oracle.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

from lbm3d_bb_b200 import Domain, abi  # noqa: E402
from oracle import oracle as orc  # noqa: E402

CHANNEL = ("inlet", "outflow", "wall", "wall", "wall", "wall")


def rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    n = np.linalg.norm(b.ravel())
    return float(np.linalg.norm((a - b).ravel()) / (n if n > 0 else 1.0))


def c1(steps=2000):
    kw = dict(collision="BGK", faces=CHANNEL, omega_p=1.0 / 0.8, face_u=[(0.04, 0, 0)] + [(0, 0, 0)] * 5,
              force_history=steps)
    out = {"workload": "c1 sphere channel 96x48x48 r=6 BGK tau=0.8 u_in=0.04", "steps": steps}
    runs = {}
    for st in ("fp64", "fp32", "fp16dev"):
        d = Domain(96, 48, 48, storage=st, **kw)
        d.add_sphere((24.0, 24.0, 24.0), 6.0)
        d.init_equilibrium()
        t0 = time.perf_counter()
        d.step(steps)
        d.synchronize()
        runs[st] = (d.force_history(1, steps), d.macros(), time.perf_counter() - t0)
        d.close()
    t0 = time.perf_counter()
    o = orc.OracleDomain(96, 48, 48, precision="fp64", **kw)
    o.add_sphere((24.0, 24.0, 24.0), 6.0)
    o.init_equilibrium()
    o.step(steps)
    fo, mo = o.force_history(1, steps), o.macros()
    out["oracle_s"] = round(time.perf_counter() - t0, 1)
    f64, m64 = runs["fp64"][0], runs["fp64"][1]
    out["fp64_vs_oracle"] = {"rho_rel_l2": rel(m64[0], mo[0]),
                             "u_rel_l2": rel(np.stack(m64[1:]), np.stack(mo[1:])),
                             "drag_lift_history_rel_l2": rel(f64[:, :3], fo[:, :3]),
                             "final_drag": float(f64[-1, 0]), "final_drag_oracle": float(fo[-1, 0])}
    for st in ("fp32", "fp16dev"):
        f = runs[st][0]
        out[f"{st}_vs_fp64"] = {"final_drag_rel_err": abs(f[-1, 0] - f64[-1, 0]) / abs(f64[-1, 0]),
                                "drag_history_rel_l2": rel(f[:, 0], f64[:, 0]),
                                "u_rel_l2": rel(np.stack(runs[st][1][1:]), np.stack(m64[1:]))}
    return out


def c2_pose(n, amp=8.0, period=2000.0, x=64.0, y0=48.0, z=48.0):
    w = 2 * math.pi / period

    def at(t):
        return abi.make_pose(center=(x, y0 + amp * math.sin(w * t), z), vel=(0.0, amp * w * math.cos(w * t), 0.0))

    return at(n - 1.0), at(n - 0.5)


def c2(steps=4000, oracle_steps=400):
    tau_p, lam = 0.56, 3.0 / 16.0
    tau_m = 0.5 + lam / (tau_p - 0.5)
    kw = dict(collision="TRT", faces=CHANNEL, omega_p=1 / tau_p, omega_m=1 / tau_m,
              face_u=[(0.03, 0, 0)] + [(0, 0, 0)] * 5, force_history=steps)

    def make(cls, **extra):
        d = cls(192, 96, 96, **kw, **extra)
        d.add_body(abi.make_body(abi.BODY_SPHERE, (64.0, 48.0, 48.0), radius=10.0, moving=True))
        d.init_equilibrium()
        return d

    out = {"workload": "c2 oscillating sphere 192x96x96 r=10 TRT tau+=0.56 Lambda=3/16 u_in=0.03", "steps": steps}
    # flags / links / populations against the oracle after every move of the first steps
    g = make(Domain, storage="fp64")
    o = make(orc.OracleDomain, precision="fp64")
    flag_mismatch, link_checks, fresh = 0, 0, 0
    prev = None
    t0 = time.perf_counter()
    for n in range(1, oracle_steps + 1):
        pn, ph = c2_pose(n)
        g.update_body(pn, ph)
        o.update_body(pn, ph)
        ms, mb = g.flags()
        mo, mbo = o.flags()
        flag_mismatch += int(not (np.array_equal(ms, mo) and np.array_equal(mb, mbo)))
        if n % 20 == 0:
            link_checks += 1
            flag_mismatch += int(not all(np.array_equal(a, b) for a, b in zip(g.links(), o.links())))
        if prev is not None:
            fresh += int(np.sum((prev == 1) & (ms == 0)))
        prev = ms
        g.step(1)
        o.step(1)
    out["oracle_s"] = round(time.perf_counter() - t0, 1)
    out["fp64_vs_oracle"] = {"steps": oracle_steps, "flag_or_link_mismatches": flag_mismatch,
                             "link_checks": link_checks, "uncovered_nodes": fresh,
                             "populations_rel_l2": rel(g.populations(), o.populations()),
                             "force_history_rel_l2": rel(g.force_history(1, oracle_steps)[:, :3],
                                                         o.force_history(1, oracle_steps)[:, :3])}
    o.close()
    g.close()
    hist = {}
    for st in ("fp64", "fp32", "fp16dev"):
        d = make(Domain, storage=st)
        t0 = time.perf_counter()
        for n in range(1, steps + 1):
            d.update_body(*c2_pose(n))
            d.step(1)
        d.synchronize()
        hist[st] = d.force_history(1, steps)
        d.check_finite()
        d.close()
    f64 = hist["fp64"]
    tail = slice(steps // 2, steps)
    for st in ("fp32", "fp16dev"):
        f = hist[st]
        out[f"{st}_vs_fp64"] = {
            "drag_history_rel_l2": rel(f[:, 0], f64[:, 0]),
            "drag_history_rel_l2_second_half": rel(f[tail, 0], f64[tail, 0]),
            "mean_drag_second_half_rel_err": abs(f[tail, 0].mean() - f64[tail, 0].mean()) / abs(f64[tail, 0].mean()),
            "lift_y_history_rel_l2": rel(f[:, 1], f64[:, 1]),
        }
    out["mean_drag_second_half_fp64"] = float(f64[tail, 0].mean())
    return out


def c3(steps=1000, n=512):
    import bench

    out = {"workload": f"c3 porous periodic {n}^3 BGK tau=0.6 g_x=1e-6", "steps": steps}
    ux = {}
    for st in ("fp64", "fp32", "fp16dev"):
        d = bench.make_domain(n, st, False, 0, None)
        d.step(steps)
        d.synchronize()
        import torch

        u = torch.empty(n ** 3, dtype=torch.float64, device="cuda")
        d.macros_into(None, u, None, None)
        fl = torch.from_numpy(d.flags()[0]).to("cuda")
        fluid = fl == 0
        ux[st] = (float(u[fluid].mean()), u)
        d.close()
    m64, u64 = ux["fp64"]
    out["mean_ux_fp64"] = m64
    for st in ("fp32", "fp16dev"):
        m, u = ux[st]
        out[f"{st}_vs_fp64"] = {"mean_ux_rel_err": abs(m - m64) / abs(m64),
                                "ux_field_rel_l2": float(((u - u64).norm() / u64.norm()).item())}
    return out


def c4(count=512, steps=1000, oracle_domains=6):
    from lbm3d_bb_b200 import sweep
    from lbm3d_bb_b200.batch import Batch

    params = sweep.sweep_params(count)
    res = {}
    for st in ("fp32", "fp64"):
        doms = [sweep.make_domain(p, storage=st, history=8) for p in params]
        with Batch(doms) as b:
            b.capture(100)
            b.replay(steps // 100)
            b.synchronize()
        fx = []
        for d in doms:
            try:
                d.check_finite()
                fx.append(float(d.force()[0]))
            except Exception:
                fx.append(float("nan"))
            d.close()
        res[st] = np.array(fx)
    ok = np.isfinite(res["fp32"]) & np.isfinite(res["fp64"])
    err = np.abs(res["fp32"][ok] - res["fp64"][ok]) / np.abs(res["fp64"][ok])
    out = {"workload": f"c4 sweep {count} domains, pressure outlet, {steps} steps", "stable": int(ok.sum()),
           "unstable_fp64": int((~np.isfinite(res["fp64"])).sum()),
           "fp32_vs_fp64_drag_rel_err": {"median": float(np.median(err)), "p95": float(np.percentile(err, 95)),
                                         "max": float(err.max())}}
    # a subset of stable domains against the oracle (smallest boxes first)
    idx = [i for i in sorted(range(count), key=lambda i: sweep.cells(params[i])) if ok[i]][:oracle_domains]
    errs = []
    for i in idx:
        o = sweep.make_domain(params[i], cls=orc.OracleDomain)
        o.step(steps)
        fo = float(o.force()[0])
        errs.append({"index": i, "oracle_fx": fo, "gpu_fp64_rel_err": abs(res["fp64"][i] - fo) / abs(fo),
                     "gpu_fp32_rel_err": abs(res["fp32"][i] - fo) / abs(fo)})
        o.close()
    out["oracle_subset"] = errs
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--only", default="c1,c2,c3,c4")
    ap.add_argument("--out", default=None)
    ap.add_argument("--quick", action="store_true", help="shorter runs (smoke of the script)")
    args = ap.parse_args()
    orc.build()
    orc.set_threads(os.cpu_count() or 1)
    q = args.quick
    jobs = {"c1": lambda: c1(200 if q else 2000), "c2": lambda: c2(200 if q else 4000, 20 if q else 400),
            "c3": lambda: c3(20 if q else 1000, 128 if q else 512), "c4": lambda: c4(16 if q else 512, 100 if q else 1000,
                                                                                   2 if q else 6)}
    results = {}
    for name in args.only.split(","):
        t0 = time.perf_counter()
        results[name] = jobs[name]()
        results[name]["wall_s"] = round(time.perf_counter() - t0, 1)
        print(json.dumps({name: results[name]}), flush=True)
    if args.out:
        Path(args.out).write_text(json.dumps(results, indent=1))


if __name__ == "__main__":
    main()
