"""What the trained network gains: held-out channel cases started from its prediction
reach steady drag in fewer steps than from rest, at the same drag (weights:
tests/golden/unet_c5.npz, trained by lbm3d_bb_b200.warmstart on seeds 0..2047)."""
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

WEIGHTS = Path(__file__).resolve().parent / "golden" / "unet_c5.npz"
HELDOUT = [100000, 100001, 100002]


def test_warm_start_reaches_steady_drag_sooner(gpu):
    import torch

    from lbm3d_bb_b200 import warmstart as W
    from lbm3d_bb_b200.unet import UNet3D, tc_status

    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        model = UNet3D.load(WEIGHTS, 0, stream)
        params = [W.case_params(s) for s in HELDOUT]
        init = W.predict(model, params)
        tc_status(stream)
        warm = W.run_to_steady_drag(params, 0, stream, init=init, drag_tol=1e-4, max_steps=60000, fallback=0.05)
        rest = W.run_to_steady_drag(params, 0, stream, init=None, drag_tol=1e-4, max_steps=60000)
    assert not warm["fell_back"].any()
    assert (warm["steps"] > 0).all() and (rest["steps"] > 0).all(), (warm["steps"], rest["steps"])
    assert (warm["steps"] < 0.7 * rest["steps"]).all(), (warm["steps"], rest["steps"])
    err = np.abs(warm["drag"] - rest["drag"]) / np.abs(rest["drag"])
    assert err.max() <= 5e-3, err


def test_bad_prediction_falls_back_to_rest(gpu):
    import torch

    from lbm3d_bb_b200 import warmstart as W

    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        p = W.case_params(100003)
        n = W.NX * W.NY * W.NZ
        rng = np.random.default_rng(0)
        bad = (np.ones(n), 0.3 * rng.standard_normal(n) * W.U_IN, np.zeros(n), np.zeros(n))
        res = W.run_to_steady_drag([p], 0, stream, init=[bad], drag_tol=1e-4, max_steps=3000, fallback=0.05)
    assert res["fell_back"].all()


def test_pipeline_end_to_end_small(gpu, tmp_path):
    import json

    from lbm3d_bb_b200 import warmstart as W

    W.main(["--train", "4", "--heldout", "2", "--epochs", "2", "--max-steps", "600", "--eval-max-steps", "3000",
            "--out", str(tmp_path)])
    res = json.loads((tmp_path / "result.json").read_text())
    assert res["train_cases"] == 4 and res["heldout"] == 2 and len(res["per_case"]) == 2
    assert np.isfinite(res["loss_last"])
    assert (tmp_path / "unet_c5.npz").exists()
