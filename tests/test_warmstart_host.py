"""Host side of the learned warm start: the case generator, the input features and the
mirror symmetry used for data augmentation and prediction averaging."""
import numpy as np
import pytest

from lbm3d_bb_b200 import warmstart as W


def test_case_table_is_deterministic_and_in_range():
    for seed in (0, 1, 100000):
        p = W.case_params(seed)
        assert p == W.case_params(seed)
        assert all(4.0 <= s <= 12.0 for s in p["semi"])
        assert 24.0 <= p["center"][0] <= 48.0
        assert W.NY / 3 <= p["center"][1] <= 2 * W.NY / 3 and W.NZ / 3 <= p["center"][2] <= 2 * W.NZ / 3
        assert 10.0 <= p["Re"] <= 100.0
        r = np.asarray(p["rot"]).reshape(3, 3)
        assert np.allclose(r @ r.T, np.eye(3)) and abs(np.linalg.det(r) - 1) < 1e-12
        assert abs(p["tau"] - (0.5 + 3 * W.U_IN * 2 * max(p["semi"]) / p["Re"])) < 1e-12


def test_features_channels():
    p = W.case_params(3)
    f = W.features(p)
    assert f.shape == (W.NZ, W.NY, W.NX, 16) and f.dtype == np.float32
    assert set(np.unique(f[..., 0])) == {0.0, 1.0}
    assert (f[..., 1][f[..., 0] == 1] <= 0).all() and (f[..., 1][f[..., 0] == 0] > -1e-3).all()
    assert np.allclose(f[..., 2], (p["Re"] - 55) / 45)
    assert np.allclose(f[0, 0, :, 3], (np.arange(W.NX) + 0.5) / W.NX)
    assert not f[..., W.N_FEATURES:].any()


@pytest.mark.parametrize("fy,fz", W.REFLECTIONS[1:])
def test_mirror_images(fy, fz):
    p = W.case_params(11)
    q = W.reflect(p, fy, fz)
    assert W.reflect(q, fy, fz)["center"] == pytest.approx(p["center"])
    assert np.allclose(W.reflect(q, fy, fz)["rot"], p["rot"])
    r = np.asarray(q["rot"]).reshape(3, 3)
    assert abs(np.linalg.det(r) - 1) < 1e-12
    m, mq = W.features(p)[..., 0], W.features(q)[..., 0]
    mm = m[:, ::-1] if fy else m
    mm = mm[::-1] if fz else mm
    # the mirrored body covers the mirrored nodes (rounding may move a grazing node)
    assert np.sum(mm != mq) <= 4 and mq.sum() > 100
    t = np.random.default_rng(0).standard_normal((W.NZ, W.NY, W.NX, 4)).astype(np.float32)
    tt = W.mirror_target(W.mirror_target(t, fy, fz), fy, fz)
    assert np.array_equal(tt, t)
    m1 = W.mirror_target(t, fy, fz)
    assert m1[0, 0, 0, 2] == (-t[-1 if fz else 0, -1 if fy else 0, 0, 2] if fy else t[-1 if fz else 0, 0, 0, 2])


def test_committed_evaluation_record_is_consistent():
    """The evaluation record of the committed weights (tests/golden/unet_c5_eval.json):
    its aggregates follow from its per-case steps and drags."""
    import json
    from pathlib import Path

    r = json.loads((Path(__file__).resolve().parent / "golden" / "unet_c5_eval.json").read_text())
    cases = r["per_case"]
    assert len(cases) == r["heldout"] == 256
    ok = [c for c in cases if c["rest_steps"] > 0 and c["warm_steps"] > 0]
    assert len(ok) == r["both_steady"]
    rest = np.array([c["rest_steps"] for c in ok], float)
    warm = np.array([c["warm_steps"] for c in ok], float)
    assert abs(rest.mean() - r["rest_steps_mean"]) < 1e-6 * rest.mean()
    assert abs(warm.mean() - r["warm_steps_mean"]) < 1e-6 * warm.mean()
    assert abs(np.mean(rest / warm) - r["step_ratio_mean"]) < 1e-9
    err = [abs(c["drag_warm"] - c["drag_rest"]) / abs(c["drag_rest"]) for c in ok]
    assert max(err) <= 5e-3  # the 0.5 % drag contract
    assert abs(r["wall_speedup"] - r["rest_set_ms"] / r["warm_set_ms"]) < 1e-9


def test_epochs_fit_the_time_budget():
    from lbm3d_bb_b200.warmstart import epochs_within

    # 2048 samples, batch 4: 512 steps per epoch at 17.9 ms -> 9.16 s per epoch
    assert epochs_within(732.0, 0.0179, 2048, 4, 200) == 79
    assert epochs_within(1e6, 0.0179, 2048, 4, 200) == 200  # capped at the wanted count
    assert epochs_within(-5.0, 0.0179, 2048, 4, 200) == 1  # at least one epoch
    assert epochs_within(10.0, 0.0, 2048, 4, 200) == 200
