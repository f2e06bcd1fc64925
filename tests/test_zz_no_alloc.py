"""lbm_get_links_noalloc: the link export for callers that cannot allocate.

Some callers of this library cannot call cudaMalloc — a host runtime that owns the
device memory pool (CUDA.jl when MainCore.jl drives the library) or a time loop that
must not pay the device-wide synchronisation of cudaMalloc/cudaFree while it rebuilds
links every step.  This entry point keeps its scratch in a fixed file-scope device
array instead.  Its CSR must equal lbm_get_links' output exactly (integer data), on
consecutive calls (the scratch keeps the previous call's contents), and lattices
above its stated maximum must be rejected with a clear error.

Kept in a file of its own that pytest collects last; it passes alone in a fresh
process and after the other tests.
"""
import ctypes

import numpy as np
import pytest

from lbm3d_bb_b200 import Domain, abi
from lbm3d_bb_b200._capi import lib
from tests import cases

pytestmark = pytest.mark.gpu


def _noalloc(d, cap):
    import torch

    ptr = torch.full((d.N + 1,), -7, dtype=torch.int32, device="cuda")
    lidx = torch.full((max(cap, 1),), -7, dtype=torch.int32, device="cuda")
    dirs = torch.full((max(cap, 1),), -7, dtype=torch.int8, device="cuda")
    nnz = ctypes.c_int64(-1)
    st = lib().lbm_get_links_noalloc(d.handle, ptr.data_ptr(), lidx.data_ptr(), dirs.data_ptr(), cap,
                                     ctypes.byref(nnz))
    n = nnz.value
    return st, n, ptr.cpu().numpy(), lidx[:n].cpu().numpy(), dirs[:n].cpu().numpy()


def _compare(d):
    ptr, lidx, dirs = d.links()
    st, n, p2, l2, d2 = _noalloc(d, len(lidx))
    assert st == abi.LBM_OK
    assert n == len(lidx)
    assert np.array_equal(ptr, p2) and np.array_equal(lidx, l2) and np.array_equal(dirs, d2)
    return n


def test_noalloc_links_equal_allocating_export_config_mode(gpu):
    d = cases.moving_sphere_trt(Domain, storage="fp32")
    counts = []
    for n in range(1, 3):  # two calls in a row, at two poses
        pn, ph = cases.sphere_pose(d, n * 7)
        d.update_body(pn, ph)
        counts.append(_compare(d))
        d.step(1)
    assert counts[0] > 0


def test_noalloc_links_equal_allocating_export_reference_mode(gpu):
    d = Domain(40, 30, 3, mode="reference", collision="BGK", omega_p=1.2, u_inf=(0.075, 0.0, 0.0))
    d.add_body(abi.make_body(abi.BODY_CYLINDER_Z, (12.5, 15.5, 0.0), radius=4.16, moving=True))
    d.init_equilibrium()
    for y in (15.5, 16.9):  # two calls in a row
        d.update_body(abi.make_pose(center=(12.5, y, 0.0)), abi.make_pose(center=(12.5, y, 0.0)))
        assert _compare(d) > 0
        d.step(1)


def test_noalloc_reports_capacity_without_overrunning(gpu):
    d = cases.sphere_channel(Domain, storage="fp32")
    ptr, lidx, dirs = d.links()
    st, n, p2, _, _ = _noalloc(d, 5)
    assert st == abi.LBM_ERR_CAPACITY and n == len(lidx)
    assert np.array_equal(ptr, p2)


def test_noalloc_large_lattice_matches_export_and_oracle(gpu, oracle_lib):
    """2,097,152 nodes: more than 1024 scan blocks, so the multi-pass carry over the
    block sums and the 64-bit block offsets run; the count is also checked against the
    CPU oracle's CSR (a bug shared by both GPU exports would not hide there)."""
    from oracle.oracle import OracleDomain

    def make(cls):
        d = cls(128, 128, 128, collision="BGK", faces=cases.PERIODIC, omega_p=1.0 / 0.6, compute_force=False)
        rng = np.random.default_rng(17)
        d.add_spheres(np.concatenate([rng.uniform(0, 128, (12, 3)), rng.uniform(4.0, 11.0, (12, 1))], axis=1))
        d.init_equilibrium()
        return d

    d = make(Domain)
    o = make(OracleDomain)
    try:
        assert d.N > 1024 * 1024
        for _ in range(2):  # two calls in a row
            n = _compare(d)
        ptr, lidx, dirs = o.links()
        st, n2, p2, l2, d2 = _noalloc(d, len(lidx))
        assert st == abi.LBM_OK and n == n2 == len(lidx) > 0
        assert np.array_equal(ptr, p2) and np.array_equal(lidx, l2) and np.array_equal(dirs, d2)
    finally:
        d.close()
        o.close()


def test_noalloc_rejects_host_memory(gpu):
    d = cases.sphere_channel(Domain, storage="fp32")
    try:
        host = np.zeros(d.N + 1, np.int32)
        nnz = ctypes.c_int64(-1)
        st = lib().lbm_get_links_noalloc(d.handle, host.ctypes.data, None, None, 0, ctypes.byref(nnz))
        assert st == abi.LBM_ERR_ARG
        assert "not" in lib().lbm_last_error(d.handle).decode()
    finally:
        d.close()


def test_noalloc_rejects_lattice_above_maximum(gpu):
    d = Domain(520, 512, 512, storage="fp16dev", compute_force=False)  # 136,314,880 > 134,217,728 nodes
    try:
        st, n, _, _, _ = _noalloc(d, 0)
        assert st == abi.LBM_ERR_CAPACITY
        assert "at most 134217728 nodes" in lib().lbm_last_error(d.handle).decode()
    finally:
        d.close()
