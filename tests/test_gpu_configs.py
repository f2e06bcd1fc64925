"""The parity contract at the workloads' full sizes, on the GPU through the C ABI.

  C1  sphere channel 96x48x48, sphere r=6 at (24,24,24), BGK tau=0.8, equilibrium inlet
      u_x=0.04, zero-gradient outflow, no-slip walls, rho=1/u=0 start, 2000 steps.
      FP64 GPU vs FP64 oracle: rho and u rel. L2 <= 1e-10, drag/lift history rel. L2
      <= 1e-9.  FP32 and FP16-deviation vs the FP64 GPU run: drag (final and mean of
      the last 500 steps) within 0.5 %, u within the stated field bounds.
  C2  oscillating sphere 192x96x96, r=10 at x=64, z=48, y_c(t)=48+8 sin(2 pi t/2000),
      TRT tau+=0.56, Lambda=3/16, inlet u_x=0.03, zero-gradient outflow, 4000 steps.
      Solid and boundary flags and the link CSR bit-exact against the oracle at every
      one of the 4000 poses; FP64 populations and forces against the oracle over the
      first 200 steps; FP32 and FP16-deviation mean drag (second half) within 0.5 % of
      the FP64 GPU run.
  C3  512^3 porous periodic box (bench workload), BGK tau=0.6, g_x=1e-6, 1000 steps:
      mean u_x of FP32 and FP16-deviation against the FP64 GPU run.
  C4  the 512-domain batched sweep (one persistent launch per step), 5000 steps:
      FP64 batch against the FP64 oracle on four domains (drag <= 1e-9), FP32 against
      FP64 on every stable domain (drag averaged over the last 200 steps within 0.5 %);
      the domains that diverge are the ones BGK cannot hold (tau < 0.52).

Stated tolerances for the reduced-precision forms (contract: drag within 0.5 % of FP64)
are the constants below; the observed errors are printed with -s.
"""
import math

import numpy as np
import pytest

from lbm3d_bb_b200 import Domain, LbmError, abi
from oracle.oracle import OracleDomain
from tests import cases
from tests.cases import rel_l2

pytestmark = pytest.mark.gpu

TOL_FIELD = 1e-10
TOL_FORCE = 1e-9
DRAG = 5e-3  # 0.5 %: drag of FP32 / FP16-deviation storage against FP64
# u (rel. L2 of the stacked velocity field) against the FP64 GPU run
U_FIELD = {"fp32": 1e-4, "fp16dev": 1e-2}
# C3: mean u_x against FP64 (u_x ~ 1e-3 there; the per-step increment g_x = 1e-6 lies
# near the FP16 resolution of the stored deviations)
C3_MEAN_UX = {"fp32": 2e-3, "fp16dev": 1e-2}

CHANNEL = ("inlet", "outflow", "wall", "wall", "wall", "wall")


def _report(name, **vals):
    print(f"\n[{name}] " + ", ".join(f"{k}={v:.3e}" if isinstance(v, float) else f"{k}={v}" for k, v in vals.items()))


# ---- C1 -----------------------------------------------------------------------------
C1_STEPS = 2000


def _c1(cls, **kw):
    d = cls(96, 48, 48, collision="BGK", faces=CHANNEL, omega_p=1.0 / 0.8, face_u=cases.face_u_inlet(0.04),
            force_history=C1_STEPS, **kw)
    d.add_sphere((24.0, 24.0, 24.0), 6.0)
    d.init_equilibrium()
    return d


@pytest.fixture(scope="module")
def c1_runs(gpu):
    out = {}
    for st in ("fp64", "fp32", "fp16dev"):
        d = _c1(Domain, storage=st)
        d.step(C1_STEPS)
        d.check_finite()
        out[st] = (d.force_history(1, C1_STEPS), d.macros())
        d.close()
    return out


def test_c1_fp64_vs_oracle(c1_runs, oracle_lib):
    o = _c1(OracleDomain, precision="fp64")
    o.step(C1_STEPS)
    fo, mo = o.force_history(1, C1_STEPS), o.macros()
    o.close()
    fg, mg = c1_runs["fp64"]
    e_rho = rel_l2(mg[0], mo[0])
    e_u = rel_l2(np.stack(mg[1:]), np.stack(mo[1:]))
    e_f = rel_l2(fg[:, :3], fo[:, :3])
    _report("C1 fp64 vs oracle", rho=e_rho, u=e_u, drag_lift_history=e_f, drag=float(fo[-1, 0]))
    assert e_rho <= TOL_FIELD and e_u <= TOL_FIELD
    assert e_f <= TOL_FORCE
    assert fo[-1, 0] > 0.0  # the flow reached the sphere: a non-trivial drag


@pytest.mark.parametrize("storage", ["fp32", "fp16dev"])
def test_c1_reduced_precision_drag(c1_runs, storage):
    f64, m64 = c1_runs["fp64"]
    f, m = c1_runs[storage]
    final = abs(f[-1, 0] - f64[-1, 0]) / abs(f64[-1, 0])
    tail = abs(f[-500:, 0].mean() - f64[-500:, 0].mean()) / abs(f64[-500:, 0].mean())
    e_u = rel_l2(np.stack(m[1:]), np.stack(m64[1:]))
    _report(f"C1 {storage} vs fp64", final_drag=final, mean_drag_last500=tail, u=e_u)
    assert final <= DRAG and tail <= DRAG
    assert e_u <= U_FIELD[storage]


# ---- C2 -----------------------------------------------------------------------------
C2_STEPS = 4000
C2_TAU_P, C2_LAMBDA = 0.56, 3.0 / 16.0


def c2_pose(n, amp=8.0, period=2000.0):
    """Poses of step n (1-based): flags at t = n-1, wall kinematics at t = n-1/2."""
    w = 2.0 * math.pi / period

    def at(t):
        return abi.make_pose(center=(64.0, 48.0 + amp * math.sin(w * t), 48.0),
                             vel=(0.0, amp * w * math.cos(w * t), 0.0))

    return at(n - 1.0), at(n - 0.5)


def _c2(cls, **kw):
    tau_m = 0.5 + C2_LAMBDA / (C2_TAU_P - 0.5)
    d = cls(192, 96, 96, collision="TRT", faces=CHANNEL, omega_p=1.0 / C2_TAU_P, omega_m=1.0 / tau_m,
            face_u=cases.face_u_inlet(0.03), **kw)
    d.add_body(abi.make_body(abi.BODY_SPHERE, (64.0, 48.0, 48.0), radius=10.0, moving=True))
    d.init_equilibrium()
    return d


def test_c2_flags_and_links_every_pose(gpu, oracle_lib):
    """Flags and links depend on the pose only: all 4000 poses, bit for bit."""
    g = _c2(Domain, storage="fp32", force_history=16)
    o = _c2(OracleDomain, precision="fp64")
    try:
        uncovered, prev, nnz_min = 0, None, None
        for n in range(1, C2_STEPS + 1):
            pn, ph = c2_pose(n)
            g.update_body(pn, ph)
            o.update_body(pn, ph)
            ms, mb = g.flags()
            mso, mbo = o.flags()
            assert np.array_equal(ms, mso), f"solid flags differ at pose {n}"
            assert np.array_equal(mb, mbo), f"boundary flags differ at pose {n}"
            lg, lo = g.links(), o.links()
            for a, b, name in zip(lg, lo, ("bb_ptr", "bb_lidxs", "bb_dirs")):
                assert np.array_equal(a, b), f"{name} differs at pose {n}"
            nnz_min = len(lg[1]) if nnz_min is None else min(nnz_min, len(lg[1]))
            if prev is not None:
                uncovered += int(np.sum((prev == 1) & (ms == 0)))
            prev = ms
        _report("C2 flags/links", poses=C2_STEPS, uncovered_nodes=uncovered, min_links=nnz_min)
        assert uncovered > 0 and nnz_min > 0
    finally:
        g.close()
        o.close()


def test_c2_fp64_vs_oracle_first_steps(gpu, oracle_lib):
    steps = 200
    g = _c2(Domain, storage="fp64", force_history=steps)
    o = _c2(OracleDomain, precision="fp64")
    try:
        for n in range(1, steps + 1):
            pn, ph = c2_pose(n)
            g.update_body(pn, ph)
            o.update_body(pn, ph)
            g.step(1)
            o.step(1)
        e_pop = rel_l2(g.populations(), o.populations())
        fg, fo = g.force_history(1, steps)[:, :3], o.force_history(1, steps)[:, :3]
        e_f = rel_l2(fg, fo)
        _report("C2 fp64 vs oracle", steps=steps, populations=e_pop, force_history=e_f)
        assert e_pop <= 1e-12
        assert e_f <= TOL_FORCE
    finally:
        g.close()
        o.close()


def test_c2_reduced_precision_mean_drag(gpu):
    hist = {}
    for st in ("fp64", "fp32", "fp16dev"):
        d = _c2(Domain, storage=st, force_history=C2_STEPS)
        for n in range(1, C2_STEPS + 1):
            d.update_body(*c2_pose(n))
            d.step(1)
        d.check_finite()
        hist[st] = d.force_history(1, C2_STEPS)
        d.close()
    f64 = hist["fp64"]
    tail = slice(C2_STEPS // 2, C2_STEPS)
    assert f64[tail, 0].mean() > 0.0
    for st in ("fp32", "fp16dev"):
        f = hist[st]
        mean_err = abs(f[tail, 0].mean() - f64[tail, 0].mean()) / abs(f64[tail, 0].mean())
        hist_err = rel_l2(f[tail, 0], f64[tail, 0])
        _report(f"C2 {st} vs fp64", mean_drag_second_half=mean_err, drag_history_second_half=hist_err)
        assert mean_err <= DRAG
        assert hist_err <= 10 * DRAG  # the oscillating drag itself, step by step


# ---- C3 -----------------------------------------------------------------------------
def test_c3_mean_ux(gpu):
    import torch

    import bench

    n, steps = 512, 1000
    mean = {}
    fluid = None
    for st in ("fp64", "fp32", "fp16dev"):
        d = bench.make_domain(n, st, False, 0, None)
        if fluid is None:
            fluid = torch.from_numpy(d.flags()[0]).to("cuda") == 0
        d.step(steps)
        d.check_finite()
        u = torch.empty(n ** 3, dtype=torch.float64, device="cuda")
        d.macros_into(None, u, None, None)
        mean[st] = float(u[fluid].mean())
        d.close()
        del u
        torch.cuda.empty_cache()
    assert mean["fp64"] > 0.0
    for st in ("fp32", "fp16dev"):
        err = abs(mean[st] - mean["fp64"]) / abs(mean["fp64"])
        _report(f"C3 {st} vs fp64", mean_ux=mean[st], mean_ux_fp64=mean["fp64"], rel_err=err)
        assert err <= C3_MEAN_UX[st]


# ---- C4 -----------------------------------------------------------------------------
def test_c4_sweep_vs_oracle(gpu, oracle_lib):
    import torch

    from lbm3d_bb_b200 import sweep
    from lbm3d_bb_b200.batch import Batch

    steps, window = 5000, 200
    params = sweep.sweep_params(512)
    fx, mean, rsd = {}, {}, {}
    for st in ("fp32", "fp64"):
        doms = [sweep.make_domain(p, storage=st, history=window) for p in params]
        try:
            with Batch(doms) as b:
                b.capture(250)
                b.replay(steps // 250)
                b.synchronize()
            last, avg, spread = [], [], []
            for d in doms:
                try:
                    d.check_finite()
                    h = d.force_history(steps - window + 1, window)[:, 0]
                    last.append(float(h[-1]))
                    avg.append(float(h.mean()))
                    spread.append(float(h.std() / abs(h.mean())))
                except LbmError:
                    last.append(float("nan"))
                    avg.append(float("nan"))
                    spread.append(float("nan"))
            fx[st], mean[st], rsd[st] = np.array(last), np.array(avg), np.array(spread)
        finally:
            for d in doms:
                d.close()
    ok = np.isfinite(fx["fp32"]) & np.isfinite(fx["fp64"])
    taus = np.array([p["tau"] for p in params])
    # the domains that diverge are the ones BGK cannot hold this close to tau = 1/2
    assert np.all(taus[~ok] < 0.52), taus[~ok]
    assert ok.sum() >= 350
    # the contract is on the drag averaged over the last 200 steps: near tau = 1/2 many wakes
    # are unsteady, and an instantaneous value of an unsteady drag differs between FP32 and
    # FP64 by the phase of the oscillation
    err32 = np.abs(mean["fp32"][ok] - mean["fp64"][ok]) / np.abs(mean["fp64"][ok])
    last32 = np.abs(fx["fp32"][ok] - fx["fp64"][ok]) / np.abs(fx["fp64"][ok])
    steady = ok & (rsd["fp64"] < 1e-3)
    _report("C4 fp32 vs fp64", stable=int(ok.sum()), steady=int(steady.sum()), median=float(np.median(err32)),
            p95=float(np.percentile(err32, 95)), max=float(err32.max()), last_step_max=float(last32.max()))
    assert err32.max() <= DRAG
    # the FP64 batch against the oracle over the full 5000 steps: the two smallest stable
    # domains of each x length
    pick = []
    for nx in sweep.SIZES_X[:2]:
        cand = [i for i in range(len(params)) if ok[i] and params[i]["nx"] == nx]
        pick += sorted(cand, key=lambda i: sweep.cells(params[i]))[:2]
    for i in pick:
        o = sweep.make_domain(params[i], cls=OracleDomain)
        o.step(steps)
        fo = float(o.force()[0])
        o.close()
        e = abs(fx["fp64"][i] - fo) / abs(fo)
        _report(f"C4 domain {i} fp64 vs oracle", nx=params[i]["nx"], ny=params[i]["ny"], drag=fo, rel_err=e)
        assert e <= TOL_FORCE
