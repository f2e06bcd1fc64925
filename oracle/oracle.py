"""ctypes wrapper of the CPU oracle (liblbm_oracle.so).

TEST INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke() and bench.py's
CPU baseline leg.  Parity status: unpinned (see lbm_oracle.h).  The class mirrors
lbm3d_bb_b200.domain.Domain method for method.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path
from typing import Optional, Sequence

import numpy as np

from lbm3d_bb_b200 import abi

HERE = Path(__file__).resolve().parent
LIB = HERE / "liblbm_oracle.so"
_lib = None


def build() -> Path:
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        L = C.CDLL(str(LIB))
        vp = C.c_void_p
        i32, i64 = C.c_int32, C.c_int64
        P = C.POINTER
        proto = {
            "orc_create": (vp, [P(abi.LbmConfig), i32]),
            "orc_destroy": (None, [vp]),
            "orc_last_error": (C.c_char_p, [vp]),
            "orc_set_threads": (i32, [i32]),
            "orc_add_body": (i32, [vp, P(abi.LbmBody)]),
            "orc_add_spheres": (i32, [vp, i32, vp]),
            "orc_update_body": (i32, [vp, P(abi.LbmPose), P(abi.LbmPose)]),
            "orc_init_equilibrium": (i32, [vp, vp, vp, vp, vp]),
            "orc_set_populations": (i32, [vp, vp]),
            "orc_step": (i32, [vp, i32]),
            "orc_step_count": (i64, [vp]),
            "orc_get_force": (i32, [vp, i64, vp]),
            "orc_get_macros": (i32, [vp, vp, vp, vp, vp]),
            "orc_get_populations": (i32, [vp, vp]),
            "orc_get_flags": (i32, [vp, vp, vp]),
            "orc_get_links": (i32, [vp, vp, vp, vp, i64, P(i64)]),
            "orc_mass": (i32, [vp, P(C.c_double)]),
        }
        for name, (res, args) in proto.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def set_threads(n: int) -> int:
    return int(lib().orc_set_threads(int(n)))


class OracleDomain:
    def __init__(self, nx: int, ny: int, nz: int, *, precision: str = "fp64", mode: str = "config",
                 collision: str = "BGK", faces: Sequence[str] = ("periodic",) * 6, omega_p: float = 1.0,
                 omega_m: Optional[float] = None, rho0: float = 1.0, face_u=None, accel=(0.0, 0.0, 0.0),
                 u_inf=(0.0, 0.0, 0.0), h: float = 1.0, compute_force: bool = True, solid_bc: str = "SBB", q: int = 19, **_ignored):
        self._L = lib()
        self.cfg = abi.make_config(nx, ny, nz, mode=abi.MODE_REFERENCE if mode == "reference" else abi.MODE_CONFIG,
                                   collision=collision, storage="fp64", faces=faces, omega_p=omega_p,
                                   omega_m=omega_m, rho0=rho0, face_u=face_u, accel=accel, u_inf=u_inf, h=h,
                                   compute_force=compute_force, solid_bc=solid_bc, q=q)
        self.shape = (int(nx), int(ny), int(nz))
        self.N = int(nx) * int(ny) * int(nz)
        self._h = self._L.orc_create(C.byref(self.cfg), 1 if precision == "fp64" else 0)
        if not self._h:
            raise RuntimeError("orc_create failed")

    def close(self):
        if getattr(self, "_h", None):
            self._L.orc_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st):
        if st != 0:
            raise RuntimeError(f"oracle status {st}: {self._L.orc_last_error(self._h).decode()}")

    def add_body(self, body):
        self._check(self._L.orc_add_body(self._h, C.byref(body)))

    def add_sphere(self, center, radius, moving=False):
        self.add_body(abi.make_body(abi.BODY_SPHERE, center, radius=radius, moving=moving))

    def add_spheres(self, xyzr):
        a = np.ascontiguousarray(xyzr, dtype=np.float64).reshape(-1, 4)
        self._check(self._L.orc_add_spheres(self._h, a.shape[0], a.ctypes.data))

    def update_body(self, pose_n, pose_half=None):
        self._check(self._L.orc_update_body(self._h, C.byref(pose_n), C.byref(pose_half) if pose_half else None))

    def init_equilibrium(self, rho=None, u=None, v=None, w=None):
        arrs = [None if a is None else np.ascontiguousarray(np.broadcast_to(a, (self.N,)), dtype=np.float64)
                for a in (rho, u, v, w)]
        self._keep = arrs
        self._check(self._L.orc_init_equilibrium(self._h, *[None if a is None else a.ctypes.data for a in arrs]))

    def set_populations(self, f, layout="soa"):
        a = np.asarray(f, dtype=np.float64)
        if layout != "soa":
            a = a.reshape(self.N, self.cfg.q).T
        a = np.ascontiguousarray(a)
        self._check(self._L.orc_set_populations(self._h, a.ctypes.data))

    def step(self, n=1):
        self._check(self._L.orc_step(self._h, int(n)))

    @property
    def step_count(self):
        return int(self._L.orc_step_count(self._h))

    def force(self, step=None):
        out = np.zeros(6)
        s = self.step_count if step is None else int(step)
        self._check(self._L.orc_get_force(self._h, s, out.ctypes.data))
        return out

    def force_history(self, first, count):
        return np.stack([self.force(first + k) for k in range(count)])

    def macros(self, dtype=np.float64):
        outs = [np.empty(self.N) for _ in range(4)]
        self._check(self._L.orc_get_macros(self._h, *[o.ctypes.data for o in outs]))
        nx, ny, nz = self.shape
        return tuple(o.astype(dtype).reshape(nz, ny, nx) for o in outs)

    def populations(self, dtype=np.float64, layout="soa"):
        out = np.empty(self.cfg.q * self.N)
        self._check(self._L.orc_get_populations(self._h, out.ctypes.data))
        out = out.reshape(self.cfg.q, self.N).astype(dtype)
        return out if layout == "soa" else np.ascontiguousarray(out.T)

    def flags(self):
        ms = np.empty(self.N, np.uint8)
        mb = np.empty(self.N, np.uint8)
        self._check(self._L.orc_get_flags(self._h, ms.ctypes.data, mb.ctypes.data))
        return ms, mb

    def links(self):
        nnz = C.c_int64()
        ptr = np.empty(self.N + 1, np.int32)
        self._L.orc_get_links(self._h, ptr.ctypes.data, None, None, 0, C.byref(nnz))
        n = nnz.value
        lidx = np.empty(max(n, 1), np.int32)
        dirs = np.empty(max(n, 1), np.int8)
        self._check(self._L.orc_get_links(self._h, ptr.ctypes.data, lidx.ctypes.data, dirs.ctypes.data, n,
                                          C.byref(nnz)))
        return ptr, lidx[:n], dirs[:n]

    def mass(self):
        m = C.c_double()
        self._check(self._L.orc_mass(self._h, C.byref(m)))
        return m.value
