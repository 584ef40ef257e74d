"""The recorded coarse-grid runs towards non-finite fields (64 x 64 x 33,
tests/golden/instability_coarse.json, made on a B200 by
tests/golden/make_instability_record.py): the reference's own build
(oracle/_ref/config0_long, config0_t400_long; the collector current printed
every 1000 steps, main.cu:227-231) and this build in FP64 from the same start.

Checked here, without a GPU:
  * both runs of each case reach non-finite fields within the recorded
    window, at the same sample (recorded: step 35,002 for config0, 71,002 for
    config0_t400, in both builds);
  * at every sample before that, the two currents agree to the six
    significant digits the reference prints ("%g"): 5e-6 relative.
"""
import json
import math

import pytest

from conftest import GOLDEN

REC = GOLDEN / "instability_coarse.json"


def first_nonfinite(currents):
    return next((k for k, c in enumerate(currents) if c is None), None)


@pytest.mark.parametrize("case", ["config0", "config0_t400"])
def test_both_builds_go_nonfinite_together(case):
    rec = json.loads(REC.read_text())[case]
    ref, ours, steps = rec["reference_current"], rec["this_build_current"], rec["steps"]
    assert len(ref) == len(ours) == len(steps) and steps[0] == 2
    kr, ko = first_nonfinite(ref), first_nonfinite(ours)
    assert kr is not None and ko is not None, (kr, ko)
    assert kr == ko, (steps[kr], steps[ko])
    for k in range(kr):
        assert math.isclose(ours[k], ref[k], rel_tol=5e-6), (steps[k], ours[k], ref[k])
