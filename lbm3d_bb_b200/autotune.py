"""Launch-shape autotuner for the step kernel.

For a lattice size, storage, collision and face set, every candidate block shape
(bx threads along x, by rows; whole warps, at most 256 threads) is timed on the
device with CUDA events over a few steps of the caller's own domain, and the fastest
is applied with ``lbm_set_launch``.  Results are cached in a JSON file keyed by GPU
name and configuration (``$LBM3D_TUNE_CACHE``, default
``~/.cache/lbm3d/launch_shapes.json``), so a shape is measured once per machine.

Tuning steps run on the caller's domain: its populations are saved before and
restored after the timing, so the field is unchanged; its step counter and force
history advance by the timed steps.
"""
from __future__ import annotations

import json
import os
from pathlib import Path
from typing import Callable, Optional, Sequence

from . import abi

FACE_NAMES = {v: k for k, v in abi.FACES.items()}


def cache_path() -> Path:
    return Path(os.environ.get("LBM3D_TUNE_CACHE", Path.home() / ".cache" / "lbm3d" / "launch_shapes.json"))


def config_key(d, device_name: str) -> str:
    c = d.cfg
    faces = ",".join(FACE_NAMES.get(int(c.face[k]), str(int(c.face[k]))) for k in range(6))
    return (f"{device_name}|{c.nx}x{c.ny}x{c.nz}|storage={int(c.storage)}|coll={int(c.collision)}|"
            f"mode={int(c.mode)}|faces={faces}")


def candidates(nx: int) -> list[tuple[int, int]]:
    """Block shapes worth timing for rows of nx cells."""
    out = []
    for bx in (32, 64, 96, 128, 256):
        if bx > max(32, -(-nx // 32) * 32):
            continue
        for threads in (128, 256):
            if threads % bx == 0:
                out.append((bx, threads // bx))
    if nx <= 256:  # whole rows, as many as fit whole warps (the default heuristic's family)
        for by in range(1, 257):
            if nx * by > 256:
                break
            if (nx * by) % 32 == 0:
                out.append((nx, by))
    return sorted(set(out))


def _load(path: Path) -> dict:
    try:
        return json.loads(path.read_text())
    except (OSError, ValueError):
        return {}


def _store(path: Path, table: dict) -> None:
    path.parent.mkdir(parents=True, exist_ok=True)
    tmp = path.with_suffix(".tmp")
    tmp.write_text(json.dumps(table, indent=1, sort_keys=True))
    tmp.replace(path)


def device_timer(d, steps: int, warmup: int) -> Callable[[], float]:
    """Milliseconds per step of the domain's current launch shape (CUDA events on its
    stream)."""
    import torch

    def run() -> float:
        d.step(warmup)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s = torch.cuda.current_stream() if d.stream is None else d.stream
        e0.record(s)
        d.step(steps)
        e1.record(s)
        e1.synchronize()
        return e0.elapsed_time(e1) / steps

    return run


def tune(d, steps: int = 10, warmup: int = 2, shapes: Optional[Sequence[tuple[int, int]]] = None,
         timer: Optional[Callable[[], float]] = None, device_name: Optional[str] = None, use_cache: bool = True,
         save_state: bool = True) -> tuple[int, int]:
    """Sets the fastest launch shape of `d` and returns it (cached per configuration)."""
    if device_name is None:
        import torch

        device_name = torch.cuda.get_device_name(d.device)
    key = config_key(d, device_name)
    path = cache_path()
    table = _load(path) if use_cache else {}
    if key in table:
        bx, by = table[key]["best"]
        d.set_launch(bx, by)
        return bx, by
    saved = None
    if save_state:
        import torch

        saved = torch.empty((19, d.N), dtype=torch.float64, device=f"cuda:{d.device}")
        d.populations_into(saved)
    run = timer or device_timer(d, steps, warmup)
    timings = {}
    for bx, by in (shapes or candidates(d.shape[0])):
        d.set_launch(bx, by)
        timings[f"{bx}x{by}"] = run()
    best = min(timings, key=timings.get)
    bx, by = (int(v) for v in best.split("x"))
    d.set_launch(bx, by)
    if saved is not None:
        d.set_populations(saved)
    if use_cache:
        table = _load(path)
        table[key] = {"best": [bx, by], "ms_per_step": timings}
        _store(path, table)
    return bx, by
