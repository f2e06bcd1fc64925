"""Batched step over many uneven domains (one persistent launch per step, CUDA graph
replay) against the same domains stepped one by one and against the CPU oracle."""
import numpy as np
import pytest

from lbm3d_bb_b200 import Domain, LbmError, abi
from lbm3d_bb_b200.batch import Batch
from oracle.oracle import OracleDomain
from tests import cases
from tests.cases import rel_l2

pytestmark = pytest.mark.gpu

# uneven sizes, some not multiples of the 128-cell work item or of a warp
SHAPES = [(24, 16, 16), (40, 16, 24), (17, 11, 13), (32, 24, 16), (9, 8, 7)]


def _member(cls, k, storage="fp64", **kw):
    nx, ny, nz = SHAPES[k]
    rng = np.random.default_rng(100 + k)
    if k == 3:  # periodic box with a body force: the forcing kernel variant
        d = cls(nx, ny, nz, collision="BGK", storage=storage, faces=cases.PERIODIC, omega_p=1.0 / 0.7,
                accel=(2e-5, 0.0, 1e-5), **kw)
        d.add_sphere((nx / 2, ny / 2, nz / 2), 3.5)
    else:
        d = cls(nx, ny, nz, collision="BGK", storage=storage, faces=cases.INLET_CHANNEL,
                omega_p=1.0 / rng.uniform(0.55, 0.9), face_u=cases.face_u_inlet(0.05), **kw)
        d.add_sphere((nx / 3, ny / 2 + 0.3, nz / 2 - 0.2), min(ny, nz) / 5)
    d.init_equilibrium()
    return d


def _members(cls, storage="fp64", **kw):
    return [_member(cls, k, storage, **kw) for k in range(len(SHAPES))]


# Batched and single launches group cells into warps differently, so a cell may take
# the inlined fast path in one and the out-of-line general path in the other; the
# two paths agree to rounding (FMA contraction may differ between them).
TOL = {"fp64": 1e-13, "fp32": 1e-6, "fp16dev": 1e-4}


def _same(a, b, steps, storage="fp64", exact=False):
    fa, fb = a.populations(), b.populations()
    if exact:
        assert np.array_equal(fa, fb), f"max diff {np.abs(fa - fb).max()}"
    else:
        assert rel_l2(fa, fb) <= TOL[storage], rel_l2(fa, fb)
    fa_, fb_ = a.force_history(1, steps)[:, :3], b.force_history(1, steps)[:, :3]
    assert np.linalg.norm(fa_ - fb_) <= 10 * TOL[storage] * np.linalg.norm(fb_) + 1e-12


@pytest.mark.parametrize("storage", ["fp64", "fp32", "fp16dev"])
def test_batch_step_matches_single_domains(gpu, storage):
    batched = _members(Domain, storage)
    single = _members(Domain, storage)
    with Batch(batched) as b:
        b.step(7)
        b.synchronize()
        assert b.launch_count == 21  # per step: two phase kernels and the counter
    for d in single:
        d.step(7)
    for a, s in zip(batched, single):
        assert a.step_count == 7
        _same(a, s, 7, storage)


def _row32(cls, k):
    """Rows of 32 cells: single launches (32 x 4 blocks) and the batch (128-cell items in
    row order) put the same cells in the same warps, so the results must agree bit for
    bit."""
    ny, nz = (8, 8) if k == 0 else (12, 5)
    faces = ("periodic", "periodic", "wall", "wall", "wall", "wall")
    d = cls(32, ny, nz, collision="BGK", storage="fp64", faces=faces, omega_p=1.0 / (0.6 + 0.1 * k),
            accel=(2e-5, 0.0, 0.0))
    d.add_sphere((11.0, ny / 2, nz / 2), 2.5)
    d.init_equilibrium()
    return d


def test_batch_bit_identical_when_warps_match(gpu):
    batched = [_row32(Domain, k) for k in range(2)]
    single = [_row32(Domain, k) for k in range(2)]
    for d in single:
        assert d.launch() == (32, 4)
    with Batch(batched) as b:
        b.step(5)
    for d in single:
        d.step(5)
    for a, s in zip(batched, single):
        _same(a, s, 5, exact=True)


def test_graph_replay_matches_steps(gpu):
    graph = _members(Domain)
    plain = _members(Domain)
    with Batch(graph) as b:
        b.capture(3)
        b.replay(3)
        b.synchronize()
    with Batch(plain) as b:
        b.step(9)
    for a, s in zip(graph, plain):
        _same(a, s, 9, exact=True)  # same kernel, same warps


def test_member_stepped_alone_between_batch_calls(gpu):
    batched = _members(Domain)
    single = _members(Domain)
    with Batch(batched) as b:
        b.capture(2)
        b.replay(1)
        batched[1].step(1)  # table follows the member (odd step count: other phase)
        b.step(3)
        batched[4].step(2)
        b.replay(2)
    counts = [2 + 3 + 4] * len(SHAPES)
    counts[1] += 1
    counts[4] += 2
    for d, n in zip(single, counts):
        d.step(n)
    for a, s, n in zip(batched, single, counts):
        assert a.step_count == n
        _same(a, s, n, "fp64")


def test_batch_vs_oracle_fp64(gpu, oracle_lib):
    g = _members(Domain)
    with Batch(g) as b:
        b.step(12)
    for k in (0, 2, 3):
        o = _member(OracleDomain, k)
        o.step(12)
        assert rel_l2(g[k].populations(), o.populations()) <= 1e-12
        fg, fo = g[k].force_history(1, 12)[:, :3], o.force_history(1, 12)[:, :3]
        assert np.linalg.norm(fg - fo) <= 1e-9 * np.linalg.norm(fo) + 1e-11


def test_batch_rejects_unsupported_members(gpu):
    a = _member(Domain, 0)
    m = cases.moving_sphere_trt(Domain, nx=24, ny=16, nz=16, r=3.0)
    with pytest.raises(LbmError) as ei:
        Batch([a, m])
    assert ei.value.status == abi.LBM_ERR_UNSUPPORTED
    c = _member(Domain, 1, storage="fp32")
    with pytest.raises(LbmError) as ei:
        Batch([a, c])
    assert ei.value.status == abi.LBM_ERR_ARG
    with pytest.raises(LbmError):
        Batch([a, a])


def test_sweep_runner_small(gpu):
    from lbm3d_bb_b200 import sweep

    params = sweep.sweep_params(6, seed=4)
    res = sweep.run_sweep(params, 40, sweep.gpu_runner("fp32", chunk=10, compare_steps=5))
    assert res["domains"] == 6
    for r in res["results"]:  # the inflow front may not have reached every sphere yet
        assert r["stable"] and np.isfinite(r["fx"])
    assert max(r["fx"] for r in res["results"]) > 0
    pr = res["per_rank"][0]
    assert pr["ms_per_step_batched_graph"] > 0 and pr["ms_per_step_one_launch_per_domain"] > 0


def _trt_member(cls, k, storage="fp64"):
    nx, ny, nz = SHAPES[k]
    tau_p = 0.56 + 0.02 * k
    tau_m = 0.5 + (3.0 / 16.0) / (tau_p - 0.5)
    d = cls(nx, ny, nz, collision="TRT", storage=storage, faces=cases.INLET_CHANNEL, omega_p=1.0 / tau_p,
            omega_m=1.0 / tau_m, face_u=cases.face_u_inlet(0.03))
    d.add_sphere((nx / 3, ny / 2, nz / 2), min(ny, nz) / 5)
    d.init_equilibrium()
    return d


@pytest.mark.parametrize("storage", ["fp64", "fp32"])
def test_batch_trt_members(gpu, oracle_lib, storage):
    """TRT domains in one batch: the same result as stepping them alone, and the FP64
    batch against the oracle."""
    batched = [_trt_member(Domain, k, storage) for k in (0, 1, 2)]
    single = [_trt_member(Domain, k, storage) for k in (0, 1, 2)]
    with Batch(batched) as b:
        b.capture(4)
        b.replay(2)
    for d in single:
        d.step(8)
    for a, s in zip(batched, single):
        _same(a, s, 8, storage)
    if storage == "fp64":
        o = _trt_member(OracleDomain, 1)
        o.step(8)
        assert rel_l2(batched[1].populations(), o.populations()) <= 1e-12
