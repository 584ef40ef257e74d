"""Pack the records of a run to saturated Nu_e into a committed fixture.

The run is bench.py's saturation workload on the reference's own default case
(122 x 122 x 101 nodes, LBM.h:31-86), from the hydrostatic state plus seeded
noise, on a B200:

  python bench.py --workload saturation --precision fp32 --record ours.json
  python bench.py --impl reference --workload saturation --sat-record ours.json \\
      --record ref.json

`ours.json` holds this build's sampled history to the step at which the
saturation criterion held; `ref.json` the reference binary's printed collector
currents over its bounded window and its time per step.  This script keeps the
summaries and the (step, Nu_e, current) history of both in
tests/golden/saturation_<name>.json:

  python tests/golden/make_saturation_record.py ours.json ref.json NAME
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

GOLDEN = Path(__file__).resolve().parent


def pack(ours: dict, ref: dict) -> dict:
    keep = ("precision", "status", "steps", "nu_e", "wall_s", "mlups", "profile_wall_s", "i0",
            "sample_every", "tol", "hold", "guard", "seed", "amp", "transits", "grid", "params")
    hist = ours["history"]
    out = {"this_build": {k: ours[k] for k in keep if k in ours},
           "this_build_history": {
               "step": [h["step"] for h in hist],
               "nu_e": [round(h["nu_e"], 9) for h in hist],
               "current": [h["current"] for h in hist],
               "kinetic_energy": [round(h["kinetic_energy"], 6) for h in hist]}}
    rkeep = ("window_steps", "window_gpu_s", "ms_per_step", "mlups", "i0", "how")
    out["reference"] = {k: ref[k] for k in rkeep if k in ref}
    # the reference's wall time projected to the step at which this run saturated
    if ours.get("status") == "saturated":
        out["reference"]["projected_to_step"] = int(ours["steps"])
        out["reference"]["value"] = round(ref["window_gpu_s"] / ref["window_steps"] * ours["steps"], 2)
    out["reference_history"] = {"step": [h["step"] for h in ref["history"]],
                                "current": [h["current"] for h in ref["history"]]}
    return out


if __name__ == "__main__":
    a, b, name = sys.argv[1], sys.argv[2], sys.argv[3]
    rec = pack(json.loads(Path(a).read_text()), json.loads(Path(b).read_text()))
    dst = GOLDEN / f"saturation_{name}.json"
    dst.write_text(json.dumps(rec))
    print("wrote", dst, dst.stat().st_size)
