"""Builds liblbm3d.so (sm_100a) in-tree with nvcc.

The library is compiled from the CUDA sources in ``csrc/``; each translation unit
gets its own flags (geometry and the reference-mode kernels are compiled without
multiply-add contraction so they round exactly as written).  The result is
``lbm3d_bb_b200/liblbm3d.so``.  Usage: ``python -m lbm3d_bb_b200.build``.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
INCLUDE = PKG.parent / "include"
LIB = PKG / "liblbm3d.so"
UNET_LIB = PKG / "libunet3d.so"
OBJ = PKG / "_build"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr"]
# per-file flags: exact rounding (no FMA contraction) where bit-exact parity is required
PER_FILE = {
    "kernels_aa.cu": [],
    "kernels_aa_fp32.cu": [],
    "kernels_aa_fp64.cu": [],
    "kernels_aa_fp16.cu": [],
    "kernels_ref.cu": ["--fmad=false"],
    "geometry.cu": ["--fmad=false"],
    "capi.cu": [],
}


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found; the CUDA toolkit is required to build liblbm3d.so")


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build(verbose: bool = False, force: bool = False) -> Path:
    """Compiles every CUDA source for sm_100a and links liblbm3d.so; returns its path."""
    OBJ.mkdir(exist_ok=True)
    headers = sorted(CSRC.glob("*.h")) + sorted(CSRC.glob("*.cuh")) + [INCLUDE / "lbm3d.h"]
    objs, jobs = [], []
    for src, flags in PER_FILE.items():
        s = CSRC / src
        o = OBJ / (s.stem + ".o")
        objs.append(o)
        if force or _stale(o, [s, *headers]):
            cmd = [nvcc(), *ARCH, *COMMON, *flags, "-c", str(s), "-o", str(o)]
            if verbose:
                cmd.insert(1, "-Xptxas=-v")
                print(" ".join(cmd), flush=True)
            jobs.append(cmd)
    # translation units compile independently: run them side by side
    workers = max(1, min(len(jobs), os.cpu_count() or 1))
    with ThreadPoolExecutor(max_workers=workers) as ex:
        for r in ex.map(lambda c: subprocess.run(c, capture_output=not verbose, text=True), jobs):
            if r.returncode != 0:
                raise RuntimeError(f"nvcc failed ({r.returncode}): {' '.join(r.args)}\n{r.stderr or ''}")
    if force or _stale(LIB, objs):
        cmd = [nvcc(), *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lcudart"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    build_unet(verbose, force)
    return LIB


def build_unet(verbose: bool = False, force: bool = False) -> Path:
    """libunet3d.so: the warm-start network's kernels (separate C ABI, include/unet3d.h)."""
    OBJ.mkdir(exist_ok=True)
    src = CSRC / "unet3d.cu"
    if force or _stale(UNET_LIB, [src, INCLUDE / "unet3d.h"]):
        cmd = [nvcc(), *ARCH, *COMMON, "-shared", str(src), "-o", str(UNET_LIB), "-lcudart"]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return UNET_LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, force="-f" in sys.argv)
    print(LIB)
