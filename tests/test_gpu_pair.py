"""Pair kernel (two x-adjacent cells per thread, two-element moves where the cells'
slots are adjacent; fully periodic boxes with nx a multiple of 128; default for
FP16-deviation storage) against the one-cell kernel and the FP64 oracle."""
import os

import numpy as np
import pytest

from lbm3d_bb_b200 import Domain
from oracle.oracle import OracleDomain
from tests import cases
from tests.cases import rel_l2

pytestmark = pytest.mark.gpu


def _porous(cls, steps, storage="fp16dev", nx=128, ny=24, nz=20, seed=5, **kw):
    rng = np.random.default_rng(seed)
    xyzr = np.concatenate([rng.uniform(0, [nx, ny, nz], (6, 3)), rng.uniform(2.0, 4.5, (6, 1))], axis=1)
    d = cls(nx, ny, nz, collision="BGK", storage=storage, faces=cases.PERIODIC, omega_p=1.0 / 0.6,
            accel=(1e-5, 0.0, 0.0), compute_force=True, **kw)
    d.add_spheres(xyzr)
    d.init_equilibrium()
    d.step(steps)
    return d


def _with_pair(enabled, fn):
    old = os.environ.get("LBM3D_PAIR")
    os.environ["LBM3D_PAIR"] = "1" if enabled else "0"
    try:
        return fn()
    finally:
        if old is None:
            del os.environ["LBM3D_PAIR"]
        else:
            os.environ["LBM3D_PAIR"] = old


TOL = {"fp16dev": 1e-4, "fp32": 1e-6, "fp64": 1e-13}


@pytest.mark.parametrize("storage", ["fp16dev", "fp32", "fp64"])
@pytest.mark.parametrize("steps", [1, 2, 9])
def test_pair_kernel_matches_one_cell_kernel(gpu, storage, steps):
    a = _with_pair(True, lambda: _porous(Domain, steps, storage))
    b = _with_pair(False, lambda: _porous(Domain, steps, storage))
    # the fast paths compute the same values; warps that fall back to the general path
    # differ between the kernels (and, for FP16, compute in absolute form): rounding level
    assert rel_l2(a.populations(), b.populations()) <= TOL[storage]
    fa, fb = a.force_history(1, steps)[:, :3], b.force_history(1, steps)[:, :3]
    assert np.linalg.norm(fa - fb) <= 10 * TOL[storage] * np.linalg.norm(fb) + 1e-11
    a.check_finite()


def test_pair_kernel_fp64_vs_oracle(gpu, oracle_lib):
    g = _with_pair(True, lambda: _porous(Domain, 12, "fp64"))
    o = _porous(OracleDomain, 12, storage="fp64")
    assert rel_l2(g.populations(), o.populations()) <= 1e-12
    fg, fo = g.force_history(1, 12)[:, :3], o.force_history(1, 12)[:, :3]
    assert np.linalg.norm(fg - fo) <= 1e-9 * np.linalg.norm(fo) + 1e-11


# Stated bounds of the pair kernels (periodic porous box, body force 1e-5 along x, 30
# steps, u_x ~ 3e-4) against the FP64 oracle: rho and u rel. L2, populations rel. L2.
PAIR_VS_ORACLE = {"fp32": {"rho": 1e-6, "u": 1e-3, "f": 1e-6},
                  "fp16dev": {"rho": 1e-4, "u": 2e-2, "f": 1e-4}}


@pytest.mark.parametrize("storage", ["fp32", "fp16dev"])
def test_pair_kernel_vs_oracle(gpu, oracle_lib, storage):
    """The bench kernels (FP32 pair kernel; FP16-deviation quad even / split odd phase)
    directly against the FP64 oracle on a periodic box with nx a multiple of 128."""
    tol = PAIR_VS_ORACLE[storage]
    g = _with_pair(True, lambda: _porous(Domain, 30, storage))
    o = _porous(OracleDomain, 30, storage="fp64")
    rg, ug, vg, wg = g.macros()
    ro, uo, vo, wo = o.macros()
    e_rho = rel_l2(rg, ro)
    e_u = rel_l2(np.stack([ug, vg, wg]), np.stack([uo, vo, wo]))
    e_f = rel_l2(g.populations(), o.populations())
    print(f"\n[{storage} pair vs fp64 oracle] rho {e_rho:.3e} u {e_u:.3e} f {e_f:.3e}")
    assert e_rho <= tol["rho"]
    assert e_u <= tol["u"]
    assert e_f <= tol["f"]
    g.check_finite()


@pytest.mark.parametrize("steps,nx", [(6, 128), (7, 128), (11, 256)])
@pytest.mark.parametrize("collision", ["BGK", "TRT"])
def test_quad_kernels_match_pair_kernels(gpu, steps, nx, collision):
    """FP16-deviation with four cells per thread in both phases (LBM3D_QUAD, default on:
    aa_quad_even_kernel; with LBM3D_QUAD_ODD=1 also aa_quad_odd_kernel with its word shifts
    exchanged through shared memory, one block per set of rows) against the pair kernels:
    same populations to storage rounding, same force history."""
    kw = {} if collision == "BGK" else {"omega_m": 1.0 / (0.5 + 0.1875 / (0.6 - 0.5))}
    var = "LBM3D_QUAD"

    def run(quad):
        old = os.environ.get(var)
        os.environ[var] = "1" if quad else "0"
        os.environ["LBM3D_QUAD_ODD"] = "1" if quad else "0"
        try:
            rng = np.random.default_rng(11)
            ny, nz = 20, 16
            xyzr = np.concatenate([rng.uniform(0, [nx, ny, nz], (6, 3)), rng.uniform(2.0, 4.5, (6, 1))], axis=1)
            d = Domain(nx, ny, nz, collision=collision, storage="fp16dev", faces=cases.PERIODIC, omega_p=1.0 / 0.6,
                       accel=(1e-5, 0.0, 0.0), compute_force=True, **kw)
            d.add_spheres(xyzr)
            d.init_equilibrium()
            d.step(steps)
            return d
        finally:
            del os.environ["LBM3D_QUAD_ODD"]
            if old is None:
                del os.environ[var]
            else:
                os.environ[var] = old

    a, b = run(True), run(False)
    try:
        assert rel_l2(a.populations(), b.populations()) <= 1e-6
        fa, fb = a.force_history(1, steps), b.force_history(1, steps)
        assert np.linalg.norm(fa - fb) <= 1e-5 * np.linalg.norm(fb) + 1e-12
    finally:
        a.close()
        b.close()


@pytest.mark.parametrize("collision", ["BGK", "TRT"])
def test_x_only_force_matches_general_force(gpu, collision):
    """FP16-deviation storage with an acceleration along x runs kernels that skip the
    exact-zero y and z source terms; a 1e-30 y-acceleration selects the general kernels.
    Same populations (to the 1e-30 terms) and force history."""
    kw = {} if collision == "BGK" else {"omega_m": 1.0 / (0.5 + 0.1875 / (0.6 - 0.5))}

    def run(gy):
        rng = np.random.default_rng(21)
        nx, ny, nz = 128, 16, 16
        xyzr = np.concatenate([rng.uniform(0, [nx, ny, nz], (5, 3)), rng.uniform(2.0, 4.0, (5, 1))], axis=1)
        d = Domain(nx, ny, nz, collision=collision, storage="fp16dev", faces=cases.PERIODIC, omega_p=1.0 / 0.6,
                   accel=(2e-5, gy, 0.0), compute_force=True, **kw)
        d.add_spheres(xyzr)
        d.init_equilibrium()
        d.step(9)
        return d

    a, b = run(0.0), run(1e-30)
    try:
        assert rel_l2(a.populations(), b.populations()) <= 1e-6
        fa, fb = a.force_history(1, 9), b.force_history(1, 9)
        assert np.linalg.norm(fa - fb) <= 1e-6 * np.linalg.norm(fb) + 1e-12
    finally:
        a.close()
        b.close()


@pytest.mark.parametrize("nx,steps", [(128, 9), (256, 10)])
@pytest.mark.parametrize("collision", ["BGK", "TRT"])
def test_fp32_shuffled_odd_phase_matches_pair_kernel(gpu, nx, steps, collision):
    """FP32 odd phase with the x-shifted directions moved as shuffled two-element words
    (LBM3D_XSHUFFLE=1: aa_pair_odd_kernel, one or two warps per row, warps with solids or
    links on the pair update) against the pair kernel: the same arithmetic on the same
    values, so the same bits."""
    kw = {} if collision == "BGK" else {"omega_m": 1.0 / (0.5 + 0.1875 / (0.6 - 0.5))}
    var = "LBM3D_XSHUFFLE"

    def run(on):
        old = os.environ.get(var)
        os.environ[var] = "1" if on else "0"
        try:
            rng = np.random.default_rng(13)
            ny, nz = 16, 12
            xyzr = np.concatenate([rng.uniform(0, [nx, ny, nz], (6, 3)), rng.uniform(2.0, 4.5, (6, 1))], axis=1)
            d = Domain(nx, ny, nz, collision=collision, storage="fp32", faces=cases.PERIODIC, omega_p=1.0 / 0.6,
                       accel=(1e-5, 0.0, 0.0), compute_force=True, **kw)
            d.add_spheres(xyzr)
            d.init_equilibrium()
            d.step(steps)
            return d
        finally:
            if old is None:
                del os.environ[var]
            else:
                os.environ[var] = old

    a, b = run(True), run(False)
    try:
        assert np.array_equal(a.populations(np.float32), b.populations(np.float32))
        # the force records are FP64 sums over links, grouped per thread and block and added
        # by atomics: a different grouping (or atomic order) moves the last bits; the force
        # bound of the parity contract applies
        fa, fb = a.force_history(1, steps), b.force_history(1, steps)
        assert np.linalg.norm(fa - fb) <= 1e-9 * np.linalg.norm(fb) + 1e-15
    finally:
        a.close()
        b.close()


@pytest.mark.parametrize("steps", [4, 7])
def test_octo_even_kernel_matches_quad_kernel(gpu, steps):
    """FP16-deviation even phase with eight cells per thread and 16-byte words (default for
    nx a multiple of 256; LBM3D_OCTO=0 keeps the four-cell kernel) against the four-cell
    kernel: the same per-cell arithmetic, so the same bits; the porous box mixes plain and
    boundary warps."""
    var = "LBM3D_OCTO"

    def run(on):
        old = os.environ.get(var)
        os.environ[var] = "1" if on else "0"
        try:
            return _porous(Domain, steps, "fp16dev", nx=256, ny=12, nz=10, seed=17)
        finally:
            if old is None:
                del os.environ[var]
            else:
                os.environ[var] = old

    a, b = run(True), run(False)
    try:
        assert np.array_equal(a.populations(np.float32), b.populations(np.float32))
        # the force records are FP64 sums over links, grouped per thread and block and added
        # by atomics: a different grouping (or atomic order) moves the last bits; the force
        # bound of the parity contract applies
        fa, fb = a.force_history(1, steps), b.force_history(1, steps)
        assert np.linalg.norm(fa - fb) <= 1e-9 * np.linalg.norm(fb) + 1e-15
    finally:
        a.close()
        b.close()


def _with_env(var, value, fn):
    old = os.environ.get(var)
    os.environ[var] = value
    try:
        return fn()
    finally:
        if old is None:
            del os.environ[var]
        else:
            os.environ[var] = old


@pytest.mark.parametrize("var,nx", [("LBM3D_QUAD_ODD", 512), ("LBM3D_QUAD_ODD", 128), ("LBM3D_QUAD_ODD", 384),
                                    ("LBM3D_QUAD_ODD", 1024)])
@pytest.mark.parametrize("steps", [2, 7])
@pytest.mark.parametrize("collision", ["BGK", "TRT"])
def test_word_odd_kernel_matches_split_kernel(gpu, var, nx, steps, collision):
    """FP16-deviation odd phase on aligned words with the x shifts exchanged between the
    threads of a row (LBM3D_QUAD_ODD=1: aa_quad_odd_kernel, four cells per thread) against
    the split pair kernel: solid cells and static links on the word path, rows next to the
    y/z wrap on the split pair update; the same per-cell arithmetic, so the same bits.  One
    to eight warps per row and one to four rows per block cover the exchange and the
    periodic x wrap."""
    kw = {} if collision == "BGK" else {"omega_m": 1.0 / (0.5 + 0.1875 / (0.6 - 0.5))}

    def run(on):
        return _with_env(var, "1" if on else "0",
                         lambda: _porous(Domain, steps, "fp16dev", nx=nx, ny=12, nz=10, seed=23, **kw))

    a, b = run(True), run(False)
    try:
        assert np.array_equal(a.populations(np.float32), b.populations(np.float32))
        # the force records are FP64 sums over links, grouped per thread and block and added
        # by atomics: a different grouping (or atomic order) moves the last bits
        fa, fb = a.force_history(1, steps), b.force_history(1, steps)
        assert np.linalg.norm(fa - fb) <= 1e-9 * np.linalg.norm(fb) + 1e-15
        a.check_finite()
    finally:
        a.close()
        b.close()


def test_word_odd_kernel_moving_body_matches_split_kernel(gpu):
    """The same comparison with a sphere moving through the periodic box: blocks with
    uncovered cells or changed links take the split pair update inside the word kernel.
    The vote that sends cells to the general path covers a block of rows in the word
    kernel and a warp in the split kernel, so a few more cells near the body run the general path,
    which computes FP16-deviation storage in absolute form: rounding level."""
    from lbm3d_bb_b200 import abi

    def run(on):
        def go():
            d = Domain(256, 24, 20, collision="BGK", storage="fp16dev", faces=cases.PERIODIC, omega_p=1.0 / 0.6,
                       accel=(1e-5, 0.0, 0.0), compute_force=True)
            d.add_body(abi.make_body(abi.BODY_SPHERE, (60.0, 12.0, 10.0), radius=5.0, moving=True))
            d.init_equilibrium()
            for n in range(1, 13):
                at = lambda t: abi.make_pose(center=(60.0 + 0.3 * t, 12.0, 10.0), vel=(0.3, 0.0, 0.0))
                d.update_body(at(n - 1.0), at(n - 0.5))
                d.step(1)
            return d
        return _with_env("LBM3D_QUAD_ODD", "1" if on else "0", go)

    a, b = run(True), run(False)
    try:
        assert rel_l2(a.populations(), b.populations()) <= TOL["fp16dev"]
        fa, fb = a.force_history(1, 12)[:, :3], b.force_history(1, 12)[:, :3]
        assert np.linalg.norm(fa - fb) <= 10 * TOL["fp16dev"] * np.linalg.norm(fb) + 1e-11
        a.check_finite()
    finally:
        a.close()
        b.close()
