"""Batch: many independent domains stepped by one persistent launch per step.

Wraps the lbm_batch_* entry points of include/lbm3d.h.  The members are ordinary
``Domain`` objects (config mode, static bodies, one device and one stream, same
storage and collision); after a batched step their forces, macros and populations
are read through the usual ``Domain`` methods.
"""
from __future__ import annotations

import ctypes as C
from typing import Sequence

from ._capi import LbmError, lib


class Batch:
    def __init__(self, domains: Sequence):
        self._L = lib()
        self.domains = list(domains)
        arr = (C.c_void_p * len(self.domains))(*[d._h.value for d in self.domains])
        h = C.c_void_p()
        st = self._L.lbm_batch_create(arr, len(self.domains), C.byref(h))
        if st != 0:
            raise LbmError(st, (self._L.lbm_global_error() or b"").decode(errors="replace"))
        self._h = h
        self._keep = arr

    def _check(self, st: int) -> None:
        if st != 0:
            raise LbmError(st, (self._L.lbm_batch_last_error(self._h) or b"").decode(errors="replace"))

    def step(self, nsteps: int = 1) -> None:
        """nsteps batched steps (three launches each: the two phase kernels and the
        counter advance)."""
        self._check(self._L.lbm_batch_step(self._h, int(nsteps)))

    def capture(self, nsteps: int) -> None:
        """Records nsteps batched steps into a CUDA graph (runs nothing)."""
        self._check(self._L.lbm_batch_capture(self._h, int(nsteps)))

    def replay(self, times: int = 1) -> None:
        """Launches the captured graph `times` times."""
        self._check(self._L.lbm_batch_replay(self._h, int(times)))

    def synchronize(self) -> None:
        self._check(self._L.lbm_batch_synchronize(self._h))

    @property
    def launch_count(self) -> int:
        return int(self._L.lbm_batch_launch_count(self._h))

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._L.lbm_batch_destroy(self._h)
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
