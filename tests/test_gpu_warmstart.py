"""The learned warm start end to end on a small grid (warmstart.py): LBM
trajectories, FNO training on the GPU, and the held-out prediction of the
state after the horizon against the plain run's.  The gain is the error of the
initial state (what the plain method has at step 0) over the error of the
prediction, both measured against the plain run at the horizon."""
import importlib.util
import math

import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu


def test_warm_start_predicts_the_horizon_state_better_than_the_start():
    spec = importlib.util.spec_from_file_location(
        "ehd_warmstart", ROOT / "ehd-convection-3d_b200" / "warmstart.py")
    W = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(W)
    res = W.main(["--train", "24", "--test", "4", "--horizon", "3000", "--epochs", "20",
                  "--relax", "200", "--grid", "16", "16", "9", "--width", "8", "--modes", "4",
                  "--layers", "2", "--hidden", "16", "--lr", "3e-3"])
    assert res["train"] == 24 and res["test"] == 4
    assert res["loss_last"] < res["loss_first"]
    assert res["gain"] > 1.5, res
    assert all(math.isfinite(x) for x in res["nu_e_warm_after_relax"])
