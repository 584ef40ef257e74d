"""Record of the coarse-grid runs towards non-finite fields (64 x 64 x 33), by
the reference's own build and by this build in FP64, from the same start.

Two cases, each from the hydrostatic column's fields plus the seeded 1e-3
velocity noise (the config0 golden start, make_golden.case_inputs):

  config0       T = 200, M = C = 10, Fe = 4000, magic parameters 1/4
                (oracle/_ref/config0_long), 40,000 steps;
  config0_t400  T = 400 with the reference's magic parameters 1/12 and 1e-6
                (oracle/_ref/config0_t400_long), 90,000 steps.

The reference binary reads the start from data_end.dat and prints the
collector current every 1000 steps (main.cu:227-231: the k-th print follows
step 2 + 1000 k); this build samples ehd_current after the same steps.  A
non-finite current is recorded as null.  Run on a GPU machine after
`python oracle/build_ref.py config0_long config0_t400_long`:

  python tests/golden/make_instability_record.py [--out FILE]
"""
from __future__ import annotations

import json
import math
import os
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

GOLDEN = Path(__file__).resolve().parent
ROOT = GOLDEN.parents[1]
sys.path.insert(0, str(GOLDEN))
sys.path.insert(0, str(ROOT / "ehd-convection-3d_b200"))
import make_golden as M  # noqa: E402

O = M.O
CASES = {
    "config0": ("config0_long", 40000,
                lambda: O.params_from_groups(64, 64, 33, 2.0, 2.0, T=200, M=10, C=10, Fe=4000)),
    "config0_t400": ("config0_t400_long", 90000,
                     lambda: O.params_from_groups(64, 64, 33, 2.0, 2.0, T=400, M=10, C=10,
                                                  Fe=4000, lambda_f=1.0 / 12.0,
                                                  lambda_g=1.0e-6)),
}


def finite_or_none(x: float):
    return x if math.isfinite(x) else None


def reference_currents(exe: Path, f: dict, nsteps: int) -> list:
    with tempfile.TemporaryDirectory() as tmp:
        M.write_data_end(Path(tmp) / "data_end.dat", f)
        r = subprocess.run([str(exe)], cwd=tmp, capture_output=True, text=True,
                           env=dict(os.environ, EHD_REF_NSTEPS=str(nsteps)), timeout=1800)
    if r.returncode != 0:
        raise RuntimeError(r.stdout[-2000:] + r.stderr[-2000:])
    out = []
    for ln in r.stdout.splitlines():
        if ln.startswith("Current = "):
            out.append(finite_or_none(float(ln.split("=")[1])))
    return out


def build_currents(ehd, p, f: dict, nsamples: int) -> list:
    out = []
    with ehd.Simulation(ehd.Params.from_dict(p.as_dict()), "fp64") as sim:
        sim.set_fields(f)
        sim.step(2)
        out.append(finite_or_none(sim.current()))
        for _ in range(nsamples - 1):
            sim.step(1000)
            out.append(finite_or_none(sim.current()))
    return out


def main(argv=None) -> None:
    import argparse

    import ehd
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=str(GOLDEN / "instability_coarse.json"))
    args = ap.parse_args(argv)
    rec = {}
    for name, (refcase, nsteps, params) in CASES.items():
        p = params()
        f, meta = M.case_inputs("config0", p)
        ref = reference_currents(ROOT / "oracle" / "_ref" / refcase / "ehd_ref", f, nsteps)
        ours = build_currents(ehd, p, f, len(ref))
        rec[name] = {"params": p.as_dict(), "nsteps": nsteps,
                     "steps": [2 + 1000 * k for k in range(len(ref))],
                     "reference_current": ref, "this_build_current": ours}
        first = lambda c: next((2 + 1000 * k for k, x in enumerate(c) if x is None), None)  # noqa
        print(name, "first non-finite sample: reference", first(ref), "this build", first(ours),
              flush=True)
    dst = Path(args.out)
    dst.write_text(json.dumps(rec))
    print("wrote", dst, dst.stat().st_size)


if __name__ == "__main__":
    main()
