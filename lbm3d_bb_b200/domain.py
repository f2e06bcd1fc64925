"""Domain: a Python handle on one liblbm3d context (one lattice on one GPU).

Thin ctypes layer over include/lbm3d.h; every method maps to one entry point and
raises ``LbmError`` on a non-zero status.  Arrays cross the boundary as numpy
(host) or as torch CUDA tensors (device, zero-copy).
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Sequence

import numpy as np

from . import abi
from ._capi import LbmError, check, lib


def _ptr(a) -> Optional[int]:
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        assert a.flags["C_CONTIGUOUS"]
        return a.ctypes.data
    return int(a.data_ptr())  # torch tensor


def _is_device(a) -> bool:
    return a is not None and not isinstance(a, np.ndarray) and getattr(a, "is_cuda", False)


class Domain:
    """One lattice (D3Q19; D3Q27 in reference mode) of nx*ny*nz nodes (x fastest) on one GPU."""

    def __init__(self, nx: int, ny: int, nz: int, *, mode: str = "config", collision: str = "BGK",
                 storage: str = "fp32", faces: Sequence[str] = ("periodic",) * 6, omega_p: float = 1.0,
                 omega_m: Optional[float] = None, rho0: float = 1.0, face_u=None, accel=(0.0, 0.0, 0.0),
                 u_inf=(0.0, 0.0, 0.0), h: float = 1.0, compute_force: bool = True, solid_bc: str = "SBB", force_history: int = 1024, q: int = 19,
                 device: int = 0, stream=None):
        self._L = lib()
        self.cfg = abi.make_config(nx, ny, nz, mode=abi.MODE_REFERENCE if mode == "reference" else abi.MODE_CONFIG,
                                   collision=collision, storage=storage, faces=faces, omega_p=omega_p,
                                   omega_m=omega_m, rho0=rho0, face_u=face_u, accel=accel, u_inf=u_inf, h=h,
                                   compute_force=compute_force, solid_bc=solid_bc, force_history=force_history, q=q)
        self.shape = (int(nx), int(ny), int(nz))
        self.N = int(nx) * int(ny) * int(nz)
        self.mode = mode
        self.device = int(device)
        self.stream = None
        handle = C.c_void_p()
        check(self._L.lbm_create(C.byref(self.cfg), int(device), C.byref(handle)))
        self._h = handle
        if stream is not None:
            self.set_stream(stream)

    # -- lifecycle -------------------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "_h", None):
            self._L.lbm_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, status: int) -> None:
        check(status, self._h)

    @property
    def handle(self) -> int:
        return self._h.value

    def set_stream(self, stream) -> None:
        """stream: a torch.cuda.Stream, a raw cudaStream_t int, or None."""
        h = getattr(stream, "cuda_stream", stream)
        self._check(self._L.lbm_set_stream(self._h, C.c_void_p(h or 0)))
        self.stream = stream if hasattr(stream, "cuda_stream") else None

    def synchronize(self) -> None:
        self._check(self._L.lbm_synchronize(self._h))

    def device_bytes(self) -> int:
        return int(self._L.lbm_device_bytes(self._h))

    def set_launch(self, bx: int, by: int) -> None:
        self._check(self._L.lbm_set_launch(self._h, int(bx), int(by)))

    def launch(self) -> tuple[int, int]:
        bx, by = C.c_int32(), C.c_int32()
        self._check(self._L.lbm_get_launch(self._h, C.byref(bx), C.byref(by)))
        return bx.value, by.value

    # -- geometry --------------------------------------------------------------------------
    def add_body(self, body: abi.LbmBody) -> None:
        self._check(self._L.lbm_add_body(self._h, C.byref(body)))

    def add_sphere(self, center, radius, moving=False) -> None:
        self.add_body(abi.make_body(abi.BODY_SPHERE, center, radius=radius, moving=moving))

    def add_spheres(self, xyzr: np.ndarray) -> None:
        a = np.ascontiguousarray(xyzr, dtype=np.float64).reshape(-1, 4)
        self._check(self._L.lbm_add_spheres(self._h, a.shape[0], a.ctypes.data))

    def update_body(self, pose_n: abi.LbmPose, pose_half: Optional[abi.LbmPose] = None) -> None:
        self._check(self._L.lbm_update_body(self._h, C.byref(pose_n), C.byref(pose_half) if pose_half else None))

    # -- state ------------------------------------------------------------------------------
    def init_equilibrium(self, rho=None, u=None, v=None, w=None) -> None:
        arrs = [None if a is None else np.ascontiguousarray(np.broadcast_to(a, (self.N,)), dtype=np.float64)
                for a in (rho, u, v, w)]
        self._check(self._L.lbm_init_equilibrium(self._h, *[_ptr(a) for a in arrs]))

    def set_populations(self, f, layout: str = "soa") -> None:
        lay = abi.LAYOUT_SOA if layout == "soa" else abi.LAYOUT_REFERENCE
        if _is_device(f):
            dt = abi.DTYPE_F64 if str(f.dtype) == "torch.float64" else abi.DTYPE_F32
            self._check(self._L.lbm_set_populations(self._h, _ptr(f), dt, lay, abi.DEVICE))
            return
        a = np.ascontiguousarray(f)
        dt = abi.DTYPE_F64 if a.dtype == np.float64 else abi.DTYPE_F32
        a = a.astype(np.float64 if dt == abi.DTYPE_F64 else np.float32, copy=False)
        self._check(self._L.lbm_set_populations(self._h, a.ctypes.data, dt, lay, abi.HOST))

    def step(self, n: int = 1) -> None:
        self._check(self._L.lbm_step(self._h, int(n)))

    # -- z-slab halo messages (faces of kind "halo") -----------------------------------------
    @property
    def halo_bytes(self) -> int:
        """Bytes of one face's message (0 without halo faces)."""
        return int(self._L.lbm_halo_bytes(self._h))

    def halo_pack(self, side: int, buf) -> None:
        """Enqueues the message of face `side` (0 z-lo, 1 z-hi) into the device tensor `buf`."""
        self._check(self._L.lbm_halo_pack(self._h, int(side), _ptr(buf)))

    def halo_unpack(self, side: int, buf) -> None:
        """Enqueues the merge of the neighbour's message `buf` on face `side`."""
        self._check(self._L.lbm_halo_unpack(self._h, int(side), _ptr(buf)))

    @property
    def step_count(self) -> int:
        return int(self._L.lbm_step_count(self._h))

    @property
    def launch_count(self) -> int:
        return int(self._L.lbm_launch_count(self._h))

    # -- outputs ----------------------------------------------------------------------------
    def force(self, step: Optional[int] = None) -> np.ndarray:
        out = np.zeros(6, dtype=np.float64)
        s = self.step_count if step is None else int(step)
        self._check(self._L.lbm_get_force(self._h, s, out.ctypes.data))
        return out

    def force_history(self, first: int, count: int) -> np.ndarray:
        out = np.zeros((count, 6), dtype=np.float64)
        self._check(self._L.lbm_get_force_history(self._h, int(first), int(count), out.ctypes.data))
        return out

    def macros(self, dtype=np.float64):
        """(rho, u, v, w) as host arrays of shape (nz, ny, nx)."""
        outs = [np.empty(self.N, dtype=dtype) for _ in range(4)]
        dt = abi.DTYPE_F64 if dtype == np.float64 else abi.DTYPE_F32
        self._check(self._L.lbm_get_macros(self._h, *[o.ctypes.data for o in outs], dt, abi.HOST))
        nx, ny, nz = self.shape
        return tuple(o.reshape(nz, ny, nx) for o in outs)

    def macros_into(self, rho, u, v, w) -> None:
        """Device export into torch CUDA tensors (float32 or float64, N elements each)."""
        ref = next(t for t in (rho, u, v, w) if t is not None)
        dt = abi.DTYPE_F64 if str(ref.dtype) == "torch.float64" else abi.DTYPE_F32
        self._check(self._L.lbm_get_macros(self._h, _ptr(rho), _ptr(u), _ptr(v), _ptr(w), dt, abi.DEVICE))

    def populations(self, dtype=np.float64, layout: str = "soa") -> np.ndarray:
        """S_n as (q, N) for layout 'soa' or (N, q) for 'reference' (f[d + q*node])."""
        lay = abi.LAYOUT_SOA if layout == "soa" else abi.LAYOUT_REFERENCE
        q = self.cfg.q
        out = np.empty(q * self.N, dtype=dtype)
        dt = abi.DTYPE_F64 if dtype == np.float64 else abi.DTYPE_F32
        self._check(self._L.lbm_get_populations(self._h, out.ctypes.data, dt, lay, abi.HOST))
        return out.reshape(q, self.N) if lay == abi.LAYOUT_SOA else out.reshape(self.N, q)

    def populations_into(self, f, layout: str = "soa") -> None:
        lay = abi.LAYOUT_SOA if layout == "soa" else abi.LAYOUT_REFERENCE
        dt = abi.DTYPE_F64 if str(f.dtype) == "torch.float64" else abi.DTYPE_F32
        self._check(self._L.lbm_get_populations(self._h, _ptr(f), dt, lay, abi.DEVICE))

    def flags(self):
        ms = np.empty(self.N, dtype=np.uint8)
        mb = np.empty(self.N, dtype=np.uint8)
        self._check(self._L.lbm_get_flags(self._h, ms.ctypes.data, mb.ctypes.data))
        return ms, mb

    def links(self):
        """(bb_ptr[N+1], bb_lidxs[nnz], bb_dirs[nnz]) in the reference's 1-based CSR."""
        nnz = C.c_int64()
        ptr = np.empty(self.N + 1, dtype=np.int32)
        st = self._L.lbm_get_links(self._h, ptr.ctypes.data, None, None, 0, C.byref(nnz))
        if st not in (abi.LBM_OK, abi.LBM_ERR_CAPACITY):
            self._check(st)
        n = nnz.value
        lidx = np.empty(max(n, 1), dtype=np.int32)
        dirs = np.empty(max(n, 1), dtype=np.int8)
        self._check(self._L.lbm_get_links(self._h, ptr.ctypes.data, lidx.ctypes.data, dirs.ctypes.data, n,
                                          C.byref(nnz)))
        return ptr, lidx[:n], dirs[:n]

    def mass(self) -> float:
        m = C.c_double()
        self._check(self._L.lbm_mass(self._h, C.byref(m)))
        return m.value

    def check_finite(self) -> None:
        self._check(self._L.lbm_check(self._h))


def read_params(path: str) -> abi.LbmParams:
    p = abi.LbmParams()
    check(lib().lbm_read_params(str(path).encode(), C.byref(p)))
    return p


def lattice(q: int = 19):
    """(cx, cy, cz, w, opp) of D3Q19 (q=19) or D3Q27 (q=27) from the library."""
    cx = np.empty(q, np.int8)
    cy = np.empty(q, np.int8)
    cz = np.empty(q, np.int8)
    w = np.empty(q, np.float32)
    op = np.empty(q, np.int8)
    check(lib().lbm_lattice(q, cx.ctypes.data, cy.ctypes.data, cz.ctypes.data, w.ctypes.data, op.ctypes.data))
    return cx, cy, cz, w, op


__all__ = ["Domain", "LbmError", "read_params", "lattice"]
