"""The recorded run to saturated Nu_e on the reference's own default case
(122 x 122 x 101 nodes, T ~ 996, M = 10, C = 10, Fe = 4000, LBM.h:31-86), from
the hydrostatic state plus seeded noise, with its reference-binary window
(tests/golden/saturation_*.json, made by tests/golden/make_saturation_record.py
from bench.py's saturation workload on a B200).

Checked here, without a GPU:
  * the saturation criterion (ehd-convection-3d_b200/saturation.py) holds at
    the recorded end and at no earlier sample;
  * over the reference's window (its collector current printed every 1000
    steps, main.cu:227-231, "%g") this build's currents at the same steps agree
    with the reference's to 2e-5 in FP64 (six printed digits) and 1e-3 in
    FP32;
  * the projected reference wall time is its time per step times the step at
    which this build's run saturated.
"""
import importlib.util
import json

import pytest

from conftest import GOLDEN, PKG

RECORDS = sorted(GOLDEN.glob("saturation_*.json"))


def saturation_module():
    spec = importlib.util.spec_from_file_location("ehd_saturation", PKG / "saturation.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


@pytest.mark.parametrize("path", RECORDS, ids=[p.stem for p in RECORDS])
def test_saturation_record(path):
    S = saturation_module()
    rec = json.loads(path.read_text())
    ours, hist = rec["this_build"], rec["this_build_history"]
    assert ours["grid"] == [122, 122, 101]
    samples = [{"step": s, "nu_e": n} for s, n in zip(hist["step"], hist["nu_e"])]
    assert samples[-1]["step"] == ours["steps"]
    if ours["status"] == "saturated":
        tol, hold, guard = ours["tol"], ours["hold"], ours["guard"]
        assert S.saturated(samples, tol, hold, guard)
        first = next(k for k in range(len(samples))
                     if S.saturated(samples[:k + 1], tol, hold, guard))
        assert first == len(samples) - 1
    ref, rhist = rec["reference"], rec["reference_history"]
    mine = dict(zip(hist["step"], hist["current"]))
    assert len(rhist["step"]) >= 10
    # FP64 against FP64 is limited by the reference's six printed digits
    tol = 2e-5 if ours["precision"] == "fp64" else 1e-3
    for s, c in zip(rhist["step"], rhist["current"]):
        assert abs(mine[s] - c) <= tol * abs(c), (s, mine[s], c)
    if ref.get("projected_to_step"):
        assert ref["projected_to_step"] == ours["steps"]
        assert ref["value"] == pytest.approx(ref["window_gpu_s"] / ref["window_steps"]
                                             * ours["steps"], rel=1e-3)
