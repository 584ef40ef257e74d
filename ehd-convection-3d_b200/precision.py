"""Storage-precision errors: the same run with FP64 populations and with FP32,
FP16 or BF16 storage, compared field by field (max-norm error relative to the
FP64 field's largest magnitude) and diagnostic by diagnostic (relative error of
Nu_e, kinetic energy and total charge), at several step counts.

Every one of the nine fields is reported on its own scale.  Two vector forms
are reported beside them: the velocity (u, v, w) and the field (Ex, Ey, Ez),
each component's error relative to the largest component of its vector.  A
component that vanishes in exact arithmetic (u and v of a flow that is still
almost z-directed, Ex and Ey of a charge that is still almost x,y-uniform)
carries only round-off and noise on its own scale, which the raw per-field
number shows and the vector number puts on the scale of the vector.  rho is
also reported against its deviation scale max|rho - rho0| ("rho_dev").

Every run starts from the same state: the hydrostatic column (its own state,
or equilibria rebuilt from its fields with --start fields) plus the seeded
velocity perturbation.  Nu_e is the two-step mean of the saturation loop.

    python ehd-convection-3d_b200/precision.py --grid 64 64 33 --steps 100 1000 5000
"""
from __future__ import annotations

import argparse
import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))

FIELDS = ("rho", "u", "v", "w", "q", "phi", "ex", "ey", "ez")
VECTORS = {"vel": ("u", "v", "w"), "E": ("ex", "ey", "ez")}
DIAGS = ("nu_e", "kinetic_energy", "total_charge")


def relerr(a: np.ndarray, b: np.ndarray) -> float:
    s = float(np.abs(b).max())
    return float(np.abs(a - b).max() / (s if s > 0 else 1.0))


def vec_err(a: dict, b: dict, comps) -> float:
    """Largest component error relative to the largest component of b."""
    s = max(float(np.abs(b[k]).max()) for k in comps)
    return max(float(np.abs(a[k] - b[k]).max()) for k in comps) / (s if s > 0 else 1.0)


def transit_steps(p, transits: float) -> int:
    """`transits` charge transit times Lz / (K V / Lz), an even number of steps."""
    n = int(round(transits * p.lz * p.lz / (p.K * p.voltage) / p.dt))
    return n + (n & 1)


def run(ehd, p, precisions, steps, seed=0, amp=1e-3, transits=16.0, start="column",
        device=0):
    """{precision: {step: {field/diagnostic: relative error against FP64}}}."""
    steps = sorted(set(int(s) for s in steps))
    n = transit_steps(p, transits)
    col, i0 = ehd.hydrostatic_column(p, n, device=device)
    prof = None
    if start == "fields":
        prof, i0 = ehd.hydrostatic_profile(p, n, device=device)
    sims = {}
    try:
        for prec in ("fp64",) + tuple(precisions):
            sim = ehd.Simulation(p, prec, device=device)
            if start == "fields":
                sim.set_state_seeded(prof, seed=seed, amp=amp)
            else:
                sim.set_state_from_column(col, seed=seed, amp=amp)
            sim.set_reference_current(i0)
            sims[prec] = sim
    finally:
        col.close()
    out = {prec: {} for prec in precisions}
    done = 0
    try:
        for s in steps:
            snap = {}
            for prec, sim in sims.items():
                d = sim.step_sampled(s - done) if s > done else sim.diagnostics()
                snap[prec] = (sim.get_fields(FIELDS), d)
            done = s
            ref_f, ref_d = snap["fp64"]
            for prec in precisions:
                f, d = snap[prec]
                row = {k: relerr(f[k], ref_f[k]) for k in FIELDS}
                for v, comps in VECTORS.items():
                    row[v] = vec_err(f, ref_f, comps)
                dev = float(np.abs(ref_f["rho"] - p.rho0).max())
                row["rho_dev"] = float(np.abs(f["rho"] - ref_f["rho"]).max()) / (dev if dev > 0 else 1.0)
                for k in DIAGS:
                    row[k] = abs(d[k] - ref_d[k]) / max(abs(ref_d[k]), 1e-300)
                row["nonfinite"] = int(d["nonfinite"])
                out[prec][s] = row
    finally:
        for sim in sims.values():
            sim.close()
    return out


def markdown(res) -> str:
    cols = FIELDS + ("vel", "E", "rho_dev") + DIAGS
    head = "| storage | step | " + " | ".join(cols) + " |"
    lines = [head, "|" + "---|" * (len(cols) + 2)]
    for prec, by_step in res.items():
        for s, row in sorted(by_step.items()):
            lines.append(f"| {prec.upper()} | {s} | " +
                         " | ".join(f"{row[c]:.1e}" for c in cols) + " |")
    return "\n".join(lines)


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--grid", type=int, nargs=3, default=(64, 64, 33), metavar=("NX", "NY", "NZ"))
    ap.add_argument("--T", type=float, default=200.0)
    ap.add_argument("--M", type=float, default=10.0)
    ap.add_argument("--C", type=float, default=10.0)
    ap.add_argument("--Fe", type=float, default=4000.0)
    ap.add_argument("--lambda-f", type=float, default=0.25)
    ap.add_argument("--lambda-g", type=float, default=0.25)
    ap.add_argument("--steps", type=int, nargs="+", default=(100, 1000, 5000))
    ap.add_argument("--precisions", nargs="+", default=("fp32", "mixed", "fp16", "bf16"),
                    choices=("fp32", "mixed", "fp16", "bf16"))
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--amp", type=float, default=1e-3)
    ap.add_argument("--transits", type=float, default=16.0)
    ap.add_argument("--start", default="column", choices=("column", "fields"))
    ap.add_argument("--out", default=None, help="write the errors (JSON) here")
    a = ap.parse_args(argv)
    import ehd
    nx, ny, nz = a.grid
    dz = 1.0 / (nz - 1)
    p = ehd.params_from_groups(nx, ny, nz, nx * dz, ny * dz, T=a.T, M=a.M, C=a.C, Fe=a.Fe,
                               lambda_f=a.lambda_f, lambda_g=a.lambda_g)
    res = run(ehd, p, a.precisions, a.steps, seed=a.seed, amp=a.amp, transits=a.transits,
              start=a.start)
    print(markdown(res), flush=True)
    if a.out:
        Path(a.out).write_text(json.dumps({k: {str(s): r for s, r in v.items()}
                                           for k, v in res.items()}, indent=1))
    return res


if __name__ == "__main__":
    main()
