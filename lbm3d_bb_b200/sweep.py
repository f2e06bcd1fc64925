"""Batched sweep: many independent channel domains of uneven sizes.

Workload (one domain per entry, numpy default_rng(seed)): Nx uniform in {48, 64, 96},
Ny = Nz uniform in {32, 48}; one fixed sphere, radius U[3, 8], centre uniform in the
central half of the box; equilibrium inlet u_x = 0.05 at x = 0, pressure outlet
(anti-bounce-back at rho0) at x = Nx-1, no-slip walls on the y/z faces; BGK with
tau = 1/2 + 3 u_x (2 r) / Re, Re log-uniform in [5, 200]; FP32 populations.  The
pressure outlet is used because a zero-gradient outflow this close behind the body
lets the wake's reverse flow grow at the outlet until the run diverges (seen at
tau = 0.8 on 48^3 boxes); tau -> 1/2 (Re near 200 at r ~ 3) is unstable with BGK
whatever the outlet, and such domains are reported as unstable.

All domains of one GPU step together: one persistent launch per step over the work
table (``Batch``), the step loop captured once in a CUDA graph and replayed.  With
several GPUs (torchrun, one process per GPU) the domains are split by cell count
(greedy, largest first) with no exchange between ranks; per-domain results are
gathered on rank 0 at the end.

Usage: python -m lbm3d_bb_b200.sweep [--count 512 --steps 5000 ...]
"""
from __future__ import annotations

import argparse
import json
import math
import os
import time
from typing import Callable, Optional, Sequence

import numpy as np

U_IN = 0.05
SIZES_X = (48, 64, 96)
SIZES_YZ = (32, 48)
CHANNEL = ("inlet", "pressure", "wall", "wall", "wall", "wall")


def sweep_params(count: int = 512, seed: int = 4) -> list[dict]:
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        nx = int(rng.choice(SIZES_X))
        n = int(rng.choice(SIZES_YZ))
        r = float(rng.uniform(3.0, 8.0))
        c = (float(rng.uniform(nx / 4, 3 * nx / 4)), float(rng.uniform(n / 4, 3 * n / 4)),
             float(rng.uniform(n / 4, 3 * n / 4)))
        re = float(math.exp(rng.uniform(math.log(5.0), math.log(200.0))))
        tau = 0.5 + 3.0 * U_IN * (2.0 * r) / re
        out.append({"index": k, "nx": nx, "ny": n, "nz": n, "r": r, "center": c, "Re": re, "tau": tau})
    return out


def cells(p: dict) -> int:
    return p["nx"] * p["ny"] * p["nz"]


def partition(params: Sequence[dict], world: int) -> list[list[int]]:
    """Domain indices per rank: largest first onto the least-loaded rank (ties: lower
    rank).  Every rank's list is in ascending index order."""
    load = [0] * world
    parts: list[list[int]] = [[] for _ in range(world)]
    for k in sorted(range(len(params)), key=lambda i: (-cells(params[i]), i)):
        r = min(range(world), key=lambda j: (load[j], j))
        parts[r].append(k)
        load[r] += cells(params[k])
    return [sorted(p) for p in parts]


def make_domain(p: dict, cls=None, storage: str = "fp32", history: int = 64, **kw):
    if cls is None:
        from .domain import Domain as cls  # noqa: N813
    d = cls(p["nx"], p["ny"], p["nz"], collision="BGK", storage=storage, faces=CHANNEL,
            omega_p=1.0 / p["tau"], face_u=[(U_IN, 0.0, 0.0)] + [(0.0, 0.0, 0.0)] * 5, compute_force=True,
            force_history=history, **kw)
    d.add_sphere(p["center"], p["r"])
    d.init_equilibrium()
    return d


def drag_coefficient(fx: float, r: float) -> float:
    return fx / (0.5 * U_IN * U_IN * math.pi * r * r)


def gpu_runner(storage: str = "fp32", chunk: int = 100, compare_steps: int = 50, device: int = 0):
    """Runs one rank's domains on its GPU; returns per-domain results and timings."""

    def run(params: Sequence[dict], steps: int) -> dict:
        import torch

        from .batch import Batch
        from .domain import LbmError

        torch.cuda.set_device(device)
        stream = torch.cuda.Stream(device=device)
        doms = [make_domain(p, storage=storage, device=device, stream=stream) for p in params]
        n_cells = sum(cells(p) for p in params)
        batch = Batch(doms)
        k = max(1, min(chunk, steps))
        reps = max(1, steps // k)
        batch.capture(k)
        batch.replay(1)  # warm-up (counts toward the steps)
        batch.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        batch.replay(reps)
        e1.record(stream)
        e1.synchronize()
        ms_graph = e0.elapsed_time(e1) / (reps * k)
        done = (reps + 1) * k
        # same domains, one launch per domain and step
        m = max(1, compare_steps)
        e0.record(stream)
        for _ in range(m):
            for d in doms:
                d.step(1)
        e1.record(stream)
        e1.synchronize()
        ms_single = e0.elapsed_time(e1) / m
        done += m
        results = []
        for p, d in zip(params, doms):
            ok = True
            try:
                d.check_finite()
            except LbmError:
                ok = False
            fx = float(d.force()[0]) if ok else float("nan")
            results.append({"index": p["index"], "steps": done, "stable": ok, "fx": fx,
                            "cd": drag_coefficient(fx, p["r"]) if ok else float("nan")})
        batch.close()
        for d in doms:
            d.close()
        return {"results": results, "cells": n_cells, "ms_per_step_batched_graph": ms_graph,
                "ms_per_step_one_launch_per_domain": ms_single, "launches_per_step_batched": 3,
                "launches_per_step_single": len(doms)}

    return run


def run_sweep(params: Sequence[dict], steps: int, runner: Callable, rank: int = 0, world: int = 1,
              dist=None) -> Optional[dict]:
    """Shards `params` over the ranks, runs this rank's part with `runner` and gathers
    the per-domain results on rank 0 (None on the other ranks)."""
    mine = [params[i] for i in partition(params, world)[rank]]
    t0 = time.perf_counter()
    out = runner(mine, steps)
    out["wall_s"] = time.perf_counter() - t0
    out["rank"] = rank
    if dist is not None and world > 1:
        gathered = [None] * world if rank == 0 else None
        dist.gather_object(out, gathered, dst=0)
        if rank != 0:
            return None
        parts = gathered
    else:
        parts = [out]
    results = sorted((r for p in parts for r in p["results"]), key=lambda r: r["index"])
    return {"domains": len(results), "results": results, "per_rank": [{k: v for k, v in p.items() if k != "results"}
                                                                       for p in parts]}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--count", type=int, default=512)
    ap.add_argument("--steps", type=int, default=5000)
    ap.add_argument("--seed", type=int, default=4)
    ap.add_argument("--chunk", type=int, default=100, help="steps per captured graph")
    ap.add_argument("--compare-steps", type=int, default=50)
    ap.add_argument("--storage", default="fp32")
    ap.add_argument("--out", default=None)
    args = ap.parse_args(argv)
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as tdist

        tdist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
        dist = tdist
    params = sweep_params(args.count, args.seed)
    res = run_sweep(params, args.steps, gpu_runner(args.storage, args.chunk, args.compare_steps, local), rank, world,
                    dist)
    if rank == 0:
        pr = res["per_rank"]
        ms_g = max(p["ms_per_step_batched_graph"] for p in pr)
        ms_s = max(p["ms_per_step_one_launch_per_domain"] for p in pr)
        total = sum(p["cells"] for p in pr)
        summary = {"domains": res["domains"], "cells": total, "ranks": world,
                   "ms_per_step_batched_graph": round(ms_g, 4), "ms_per_step_one_launch_per_domain": round(ms_s, 4),
                   "speedup": round(ms_s / ms_g, 3), "mlups_batched": round(total / (ms_g * 1e-3) / 1e6, 1),
                   "unstable_domains": [r["index"] for r in res["results"] if not r["stable"]]}
        print(json.dumps(summary), flush=True)
        if args.out:
            with open(args.out, "w") as f:
                json.dump({"summary": summary, **res}, f)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
