#!/usr/bin/env python
"""Throughput of the fused D3Q19 step on B200 (MLUPS and HBM roofline fraction).

Workload (the roofline configuration): 512^3 D3Q19, BGK tau=0.6, fully periodic,
uniform body force g_x=1e-6 (Guo), porous solid of 200 overlapping spheres
(radius U[6,16], centres U[0,512)^3, numpy default_rng(3)), initial rho=1, u=0,
FP32 populations.  One step = one fused AA-pattern kernel launch over all cells (two x-adjacent
cells per thread for FP32 and FP16-deviation storage on this box).
MLUPS counts every cell, solid included (the reference's measure_Mlups,
Utilities.jl:903-926).

Usage: python bench.py [--gpus N --steps K --warmup W] [--impl reference]
Multi-GPU (torchrun): every rank runs its own 512^3 replica (the single-domain
path does not shard); the value is the sum over ranks with the max-over-ranks time.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "MLUPS (D3Q19 fused step, all cells)"
UNIT = "MLUPS"
TAU = 0.6
GX = 1e-6
NSPHERES = 200
SEED = 3
BYTES_PER_CELL = {"fp32": 2 * 19 * 4 + 1, "fp16dev": 2 * 19 * 2 + 1, "fp64": 2 * 19 * 8 + 1}
DTYPE = {"fp32": "f32", "fp16dev": "f16 storage / f32 compute", "fp64": "f64"}


def sphere_table(n: int, count: int, seed: int = SEED) -> np.ndarray:
    rng = np.random.default_rng(seed)
    c = rng.uniform(0.0, float(n), (count, 3))
    r = rng.uniform(6.0, 16.0, (count, 1))
    return np.concatenate([c, r], axis=1)


def workload(n: int) -> dict:
    return {
        "workload": f"porous periodic {n}^3 D3Q19 BGK tau={TAU} g_x={GX:g}, "
                    f"{max(1, round(NSPHERES * (n / 512) ** 3))} spheres r~U[6,16] seed {SEED}",
        "nx": n, "ny": n, "nz": n, "collision": "BGK", "tau": TAU, "body_force": [GX, 0.0, 0.0],
        "parallelism": "replicas (one independent domain per GPU)",
        "l2": "inputs larger than L2: population array >> 126 MB, no flush between steps",
    }


def load_peaks() -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except Exception:
            pass
    return 6650.0, "fallback"


def step_kernel(storage: str, n: int) -> str:
    """The kernel a fully periodic n^3 box runs (two cells per thread for FP32 and
    FP16-deviation when n is a multiple of 128; FP16-deviation odd steps run the split
    variant)."""
    pair = n % 128 == 0 and storage != "fp64"
    env = os.environ.get("LBM3D_PAIR")
    if env is not None:
        pair = n % 128 == 0 and env == "1"
    if not pair:
        return "aa_step_kernel"
    if storage == "fp16dev":
        quad = os.environ.get("LBM3D_QUAD") != "0"
        octo = quad and n % 256 == 0 and os.environ.get("LBM3D_OCTO") != "0"
        even = "aa_octo_even_kernel" if octo else ("aa_quad_even_kernel" if quad else "aa_pair_kernel")
        return even + " / aa_pair_split_kernel"
    return "aa_pair_kernel"


def profiled_traffic(storage: str, n: int):
    """DRAM bytes per cell of the step kernel from the committed ncu summary."""
    kind = "step" if step_kernel(storage, n) == "aa_step_kernel" else "pair"
    f = ROOT / "profiles" / f"aa_{kind}_{storage}_porous.txt"
    if not f.exists():
        return None
    for line in f.read_text().splitlines():
        if line.startswith("dram_bytes_per_cell:"):
            return float(line.split(":", 1)[1].split()[0]) * n ** 3
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.idx = device_index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "50",
                 "-i", str(self.idx)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        time.sleep(0.15)
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()
                out = ""
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self) -> dict:
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in getattr(self, "lines", []):
            parts = [p.strip() for p in l.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def make_domain(n: int, storage: str, compute_force: bool, device: int, stream):
    from lbm3d_bb_b200 import Domain

    d = Domain(n, n, n, collision="BGK", storage=storage, faces=("periodic",) * 6, omega_p=1.0 / TAU,
               accel=(GX, 0.0, 0.0), compute_force=compute_force, force_history=4096, device=device, stream=stream)
    d.add_spheres(sphere_table(n, max(1, round(NSPHERES * (n / 512) ** 3))))
    d.init_equilibrium()
    return d


def solid_count(d) -> int:
    return int(d.flags()[0].sum())


def time_device(d, stream, steps: int, warmup: int, dist, device_index: int):
    """W untimed steps, then K steps between CUDA events on the library's stream."""
    import torch

    d.step(warmup)
    d.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    l0 = d.launch_count
    with ClockSampler(device_index) as clk:
        ev0.record(stream)
        d.step(steps)
        ev1.record(stream)
        ev1.synchronize()
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    if dist is not None:
        dist.barrier()
    return ms, d.launch_count - l0, clk.summary()


def time_e2e(n: int, storage: str, steps: int, warmup: int, device: int, stream, dist):
    """Through the public API with host data every step: the body kinematics go in
    (lbm_update_body, host structs) and the step's momentum-exchange force comes
    back (lbm_get_force, device->host copy + wait)."""
    import torch

    from lbm3d_bb_b200 import abi

    d = make_domain(n, storage, True, device, stream)
    pose = abi.make_pose(center=(n / 2, n / 2, n / 2))
    for _ in range(warmup):
        d.update_body(pose, pose)
        d.step(1)
        d.force()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    ev0.record(stream)
    last = None
    for _ in range(steps):
        d.update_body(pose, pose)
        d.step(1)
        last = d.force()
    ev1.record(stream)
    ev1.synchronize()
    ms = ev0.elapsed_time(ev1)
    d.close()
    h2d = 2 * C_sizeof_pose()
    d2h = 8 * 32 * 8  # one force record (32 cache lines of 8 doubles)
    return ms, h2d, d2h, last


def time_moving_body(steps: int, warmup: int, device: int, stream, dist, storage: str = "fp32"):
    """The oscillating-sphere channel (192x96x96, TRT tau+ 0.56, Lambda 3/16, inlet u_x 0.03,
    sphere r 10 at x 64, z 48, y_c(t) = 48 + 8 sin(2 pi t / 2000)) through the public API: every
    step the host evaluates the motion law and passes the two poses (lbm_update_body), and the
    step rebuilds the moving body's flags and links in its box, refills the uncovered nodes
    and runs the face-aware step kernel (the reference's per-step motion!, Motion.jl:41-122,
    plus collision through the momentum exchange)."""
    import torch

    from lbm3d_bb_b200 import Domain, abi

    tau_p, lam = 0.56, 3.0 / 16.0
    d = Domain(192, 96, 96, collision="TRT", storage=storage, faces=("inlet", "outflow", "wall", "wall", "wall", "wall"),
               omega_p=1.0 / tau_p, omega_m=1.0 / (0.5 + lam / (tau_p - 0.5)),
               face_u=[(0.03, 0.0, 0.0)] + [(0.0, 0.0, 0.0)] * 5, force_history=4096, device=device, stream=stream)
    d.add_body(abi.make_body(abi.BODY_SPHERE, (64.0, 48.0, 48.0), radius=10.0, moving=True))
    d.init_equilibrium()
    w = 2.0 * math.pi / 2000.0

    def poses(n):
        def at(t):
            return abi.make_pose(center=(64.0, 48.0 + 8.0 * math.sin(w * t), 48.0),
                                 vel=(0.0, 8.0 * w * math.cos(w * t), 0.0))
        return at(n - 1.0), at(n - 0.5)

    n = 0
    for _ in range(warmup):
        n += 1
        d.update_body(*poses(n))
        d.step(1)
    d.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    l0 = d.launch_count
    ev0.record(stream)
    for _ in range(steps):
        n += 1
        d.update_body(*poses(n))
        d.step(1)
    ev1.record(stream)
    ev1.synchronize()
    ms = ev0.elapsed_time(ev1)
    launches = d.launch_count - l0
    d.check_finite()
    d.close()
    return ms, launches, 192 * 96 * 96


def C_sizeof_pose() -> int:
    import ctypes

    from lbm3d_bb_b200 import abi

    return ctypes.sizeof(abi.LbmPose)


CPU_N = 256        # edge of the CPU sample cube (same sphere density as the 512^3 box)
CPU_WARMUP = 2     # untimed steps before the timed runs
CPU_STEPS = 6      # steps per timed run
CPU_REPEATS = 5    # timed runs; the best is reported (the host cores are shared: the fastest
                   # run is the one least disturbed by other work), the median beside it


def cpu_sample(n: int = CPU_N, steps: int = CPU_STEPS, repeats: int = CPU_REPEATS, warmup: int = CPU_WARMUP) -> dict:
    """The CPU restatement (oracle, FP32, all host threads) on the fixed sample cube:
    `warmup` untimed steps, then `repeats` timed runs of `steps` steps; best and median MLUPS.
    Runs in a process without torch or CUDA (see cpu_baseline)."""
    from oracle import oracle as orc

    orc.build()
    avail = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    cores = orc.set_threads(avail)
    spheres = max(1, round(NSPHERES * (n / 512) ** 3))
    o = orc.OracleDomain(n, n, n, precision="fp32", collision="BGK", faces=("periodic",) * 6, omega_p=1.0 / TAU,
                         accel=(GX, 0.0, 0.0), compute_force=False)
    o.add_spheres(sphere_table(n, spheres))
    o.init_equilibrium()
    o.step(warmup)
    runs = []
    for _ in range(repeats):
        t0 = time.perf_counter()
        o.step(steps)
        runs.append(n ** 3 * steps / (time.perf_counter() - t0) / 1e6)
    o.close()
    med = statistics.median(runs)
    return {"value": round(max(runs), 3), "median": round(med, 3), "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{n}^3 periodic porous cube ({spheres} spheres, same density), FP32, {warmup} warm-up steps, "
                      f"best of {repeats} runs of {steps} steps ({', '.join(f'{r:.1f}' for r in runs)} MLUPS)",
            "n": n, "runs": [round(r, 3) for r in runs]}


def cpu_baseline() -> dict:
    """cpu_sample in a fresh interpreter that loads neither torch nor CUDA, so that both
    arms time the same sample under the same conditions."""
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    env.setdefault("OMP_PROC_BIND", "close")  # one thread per core, kept in place
    env.setdefault("OMP_PLACES", "cores")
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--cpu-sample"], capture_output=True, text=True,
                       env=env, timeout=900)
    if r.returncode != 0:
        raise RuntimeError(f"CPU sample failed ({r.returncode}): {r.stderr[-2000:]}")
    return json.loads(r.stdout.strip().splitlines()[-1])


def run_reference_arm(args, rank: int, world: int):
    if rank != 0:
        return
    base = cpu_baseline()
    n = base.pop("n")
    base.pop("runs", None)
    line = {
        "impl": "reference", "metric": METRIC, "value": base["value"], "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(n ** 3 / (base["value"] * 1e6) * 1e3, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": dict(workload(n), sampled_for=workload(args.size)["workload"]),
        "cpu_baseline": base,
        "e2e": {"value": base["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "the reference has no CPU path (CuArray{Float32} kernels, julia absent): the CPU restatement of "
                "its step is timed on the host cores, on a fixed sample cube of the same workload",
    }
    print(json.dumps(line), flush=True)


def roofline(storage, ms_per_launch, n_cells, n_solid, peak, peak_kind, traffic):
    bytes_launch = (n_cells - n_solid) * BYTES_PER_CELL[storage] + n_solid * 1
    achieved = bytes_launch / (ms_per_launch * 1e-3) / 1e9
    n = round(n_cells ** (1.0 / 3.0))
    return {"kernel": step_kernel(storage, n), "bound": "hbm", "achieved": round(achieved, 1), "peak": peak,
            "unit": "GB/s",
            "frac": round(achieved / peak, 4), "peak_kind": peak_kind,
            "traffic": None if traffic is None else round(traffic, 0),
            "algorithmic_bytes_per_launch": bytes_launch}


def main():
    global GX
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--size", type=int, default=512)
    ap.add_argument("--storage", default="fp32", choices=["fp32", "fp16dev", "fp64"])
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-secondary", action="store_true")
    ap.add_argument("--no-moving", action="store_true", help="skip the moving-body channel line")
    ap.add_argument("--gx", type=float, default=GX, help="body acceleration along x (workload default 1e-6)")
    ap.add_argument("--cpu-sample", action="store_true", help=argparse.SUPPRESS)
    args = ap.parse_args()
    if args.cpu_sample:  # child process of cpu_baseline(): no torch, no CUDA
        print(json.dumps(cpu_sample()), flush=True)
        return
    args.warmup = max(3, args.warmup)
    GX = args.gx

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        run_reference_arm(args, rank, world)
        return

    import torch

    from lbm3d_bb_b200 import build

    # one rank brings the in-tree libraries up to date (a no-op when they are current);
    # the others wait for it in the process-group rendezvous
    if rank == 0:
        build.build()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as tdist

        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        dist = tdist
    stream = torch.cuda.Stream(device=local)
    dev_index = local
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    if vis:
        try:
            dev_index = int(vis.split(",")[local])
        except ValueError:
            pass

    peak, peak_kind = load_peaks()
    n = args.size
    N = n ** 3

    d = make_domain(n, args.storage, False, local, stream)
    n_solid = solid_count(d)
    ms, launches, clocks = time_device(d, stream, args.steps, args.warmup, dist, dev_index)
    d.check_finite()
    d.close()
    del d
    torch.cuda.empty_cache()
    if dist is not None:
        t = torch.tensor([ms], device=f"cuda:{local}", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    ms_step = ms / args.steps
    value = world * N * args.steps / (ms * 1e-3) / 1e6

    secondary = None
    if not args.no_secondary and args.storage == "fp32":
        d2 = make_domain(n, "fp16dev", False, local, stream)
        ms2, _, _ = time_device(d2, stream, args.steps, args.warmup, dist, dev_index)
        d2.close()
        del d2
        torch.cuda.empty_cache()
        if dist is not None:
            t = torch.tensor([ms2], device=f"cuda:{local}", dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms2 = float(t.item())
        v2 = world * N * args.steps / (ms2 * 1e-3) / 1e6
        secondary = {"storage": "fp16dev", "value": round(v2, 1), "unit": UNIT,
                     "ms_per_step": round(ms2 / args.steps, 4), "speedup_vs_fp32": round(v2 / value, 3),
                     "roofline": roofline("fp16dev", ms2 / args.steps, N, n_solid, peak, peak_kind,
                                          profiled_traffic("fp16dev", n))}

    e2e = None
    if not args.no_e2e:
        e_steps = max(10, min(args.steps, 100))
        ms_e, h2d, d2h, _ = time_e2e(n, args.storage, e_steps, args.warmup, local, stream, dist)
        if dist is not None:
            t = torch.tensor([ms_e], device=f"cuda:{local}", dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms_e = float(t.item())
        e2e = {"value": round(world * N * e_steps / (ms_e * 1e-3) / 1e6, 1), "unit": UNIT,
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "steps": e_steps,
               "path": "Domain.update_body (host pose structs) -> lbm_step(1) -> lbm_get_force (D2H + wait), "
                       "force accumulation on"}
        torch.cuda.empty_cache()

    moving = None
    if not args.no_moving:
        m_steps = max(20, min(4 * args.steps, 400))
        ms_m, l_m, cells_m = time_moving_body(m_steps, args.warmup, local, stream, dist)
        if dist is not None:
            t = torch.tensor([ms_m], device=f"cuda:{local}", dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms_m = float(t.item())
        moving = {"workload": "oscillating sphere channel 192x96x96 D3Q19 TRT tau+=0.56 Lambda=3/16, r=10, "
                              "y_c(t)=48+8 sin(2 pi t/2000), inlet u_x=0.03, FP32",
                  "value": round(world * cells_m * m_steps / (ms_m * 1e-3) / 1e6, 1), "unit": UNIT,
                  "ms_per_step": round(ms_m / m_steps, 4), "steps": m_steps,
                  "launches_per_step": round(l_m / m_steps, 2),
                  "path": "host poses -> lbm_update_body -> lbm_step(1): moving-body flags and links in the "
                          "body's box, refill, face-aware step kernel"}
        torch.cuda.empty_cache()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline()
        cpu.pop("n", None)
        cpu.pop("runs", None)

    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms_step, 4), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": DTYPE[args.storage], "data": "synthetic", "config": workload(n),
            "roofline": roofline(args.storage, ms_step, N, n_solid, peak, peak_kind,
                                 profiled_traffic(args.storage, n)),
            "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": int(launches), "clocks": clocks,
            "solid_fraction": round(n_solid / N, 5),
        }
        if secondary:
            line["fp16dev"] = secondary
        if moving:
            line["moving_body"] = moving
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
