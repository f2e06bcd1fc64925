"""Loads liblbm3d.so and declares the prototypes of include/lbm3d.h.

There is no fallback: if the library is missing the import fails with a message
naming the build command.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

from .abi import ABI_VERSION, LbmBody, LbmConfig, LbmParams, LbmPose

LIB_PATH = Path(os.environ.get("LBM3D_LIB", Path(__file__).resolve().parent / "liblbm3d.so"))

_lib = None


class LbmError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"[status {status}] {message}")
        self.status = status


def lib() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(
            f"{LIB_PATH} is missing: the CUDA library is required (build it with `python -m lbm3d_bb_b200.build`)"
        )
    L = C.CDLL(str(LIB_PATH))
    P = C.POINTER
    vp = C.c_void_p
    i32, i64, f64 = C.c_int32, C.c_int64, C.c_double
    proto = {
        "lbm_abi_version": (i32, []),
        "lbm_status_string": (C.c_char_p, [i32]),
        "lbm_global_error": (C.c_char_p, []),
        "lbm_read_params": (i32, [C.c_char_p, P(LbmParams)]),
        "lbm_lattice": (i32, [i32, vp, vp, vp, vp, vp]),
        "lbm_create": (i32, [P(LbmConfig), i32, P(vp)]),
        "lbm_destroy": (i32, [vp]),
        "lbm_last_error": (C.c_char_p, [vp]),
        "lbm_set_stream": (i32, [vp, vp]),
        "lbm_synchronize": (i32, [vp]),
        "lbm_device_bytes": (i64, [vp]),
        "lbm_set_launch": (i32, [vp, i32, i32]),
        "lbm_get_launch": (i32, [vp, P(i32), P(i32)]),
        "lbm_add_body": (i32, [vp, P(LbmBody)]),
        "lbm_add_spheres": (i32, [vp, i32, vp]),
        "lbm_update_body": (i32, [vp, P(LbmPose), P(LbmPose)]),
        "lbm_init_equilibrium": (i32, [vp, vp, vp, vp, vp]),
        "lbm_set_populations": (i32, [vp, vp, i32, i32, i32]),
        "lbm_step": (i32, [vp, i32]),
        "lbm_step_count": (i64, [vp]),
        "lbm_launch_count": (i64, [vp]),
        "lbm_get_force": (i32, [vp, i64, vp]),
        "lbm_get_force_history": (i32, [vp, i64, i32, vp]),
        "lbm_get_macros": (i32, [vp, vp, vp, vp, vp, i32, i32]),
        "lbm_get_populations": (i32, [vp, vp, i32, i32, i32]),
        "lbm_get_flags": (i32, [vp, vp, vp]),
        "lbm_get_links": (i32, [vp, vp, vp, vp, i64, P(i64)]),
        "lbm_get_links_noalloc": (i32, [vp, vp, vp, vp, i64, P(i64)]),
        "lbm_halo_bytes": (i64, [vp]),
        "lbm_halo_pack": (i32, [vp, i32, vp]),
        "lbm_halo_unpack": (i32, [vp, i32, vp]),
        "lbm_mass": (i32, [vp, P(f64)]),
        "lbm_check": (i32, [vp]),
        "lbm_wait_selftest": (i32, [vp, i32]),
        "lbm_batch_create": (i32, [vp, i32, P(vp)]),
        "lbm_batch_destroy": (i32, [vp]),
        "lbm_batch_last_error": (C.c_char_p, [vp]),
        "lbm_batch_step": (i32, [vp, i32]),
        "lbm_batch_capture": (i32, [vp, i32]),
        "lbm_batch_replay": (i32, [vp, i32]),
        "lbm_batch_launch_count": (i64, [vp]),
        "lbm_batch_synchronize": (i32, [vp]),
    }
    for name, (res, args) in proto.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    if L.lbm_abi_version() != ABI_VERSION:
        raise ImportError(f"liblbm3d.so ABI {L.lbm_abi_version()} != {ABI_VERSION}")
    _lib = L
    return L


def exported_symbols() -> list[str]:
    """Names every declaration of include/lbm3d.h binds (for load tests)."""
    return [
        "lbm_abi_version", "lbm_status_string", "lbm_global_error", "lbm_read_params", "lbm_lattice",
        "lbm_create", "lbm_destroy", "lbm_last_error", "lbm_set_stream", "lbm_synchronize",
        "lbm_device_bytes", "lbm_set_launch", "lbm_get_launch", "lbm_add_body", "lbm_add_spheres",
        "lbm_update_body", "lbm_init_equilibrium", "lbm_set_populations", "lbm_step", "lbm_step_count", "lbm_launch_count",
        "lbm_get_force", "lbm_get_force_history", "lbm_get_macros", "lbm_get_populations", "lbm_get_flags",
        "lbm_get_links", "lbm_get_links_noalloc", "lbm_mass", "lbm_check", "lbm_wait_selftest",
        "lbm_batch_create", "lbm_batch_destroy", "lbm_batch_last_error", "lbm_batch_step", "lbm_batch_capture",
        "lbm_batch_replay", "lbm_batch_launch_count", "lbm_batch_synchronize",
        "lbm_halo_bytes", "lbm_halo_pack", "lbm_halo_unpack",
    ]


def check(status: int, ctx=None) -> None:
    if status == 0:
        return
    L = lib()
    msg = (L.lbm_last_error(ctx) if ctx else L.lbm_global_error()) or b""
    raise LbmError(status, msg.decode(errors="replace") or L.lbm_status_string(status).decode())
