"""Wall time to saturated Nu_e on one case, by default the reference's own
default case (LBM.h:31-86): 122 x 122 x 101 nodes, dx = dz = 1/100,
Lx = Ly = 1.22, dt = 1e-4, nu = 0.0251004, K = 2.5e-5, charge0 = 10,
D = 6.25e-5, TRT magic parameters 1/12 (f) and 1e-6 (g), i.e. T ~ 996,
M = 10, C = 10, Fe = 4000 (compute_parameters, LBM.cu:1375-1378).

The run starts from the hydrostatic state (the u = 0 steady state of the same
step on a 1 x 1 x NZ column, 16 charge transit times) broadcast over x, y plus
the seeded 1e-3 velocity perturbation (ehd_set_state_seeded), the state the
reference is given through data_end.dat for the same comparison.  It samples
the collector current every `sample_every` steps at steps 2, 2 + S, 2 + 2S, ...
(the steps at which the reference prints it, `i % printCurrent == 1`,
main.cu:227-231), Nu_e as the mean of the currents after the last two steps
over the hydrostatic current I0 (the injector makes the current alternate
with a period of two steps).

Saturation: the flow has left the hydrostatic state (|Nu_e - 1| > guard at
some sample) and |Nu_e(k) - Nu_e(k-1)| / Nu_e(k) < tol for `hold` consecutive
samples.  Without the guard the criterion is met at once near the hydrostatic
state, where Nu_e changes by less than tol per sample during the linear
growth.

    python ehd-convection-3d_b200/saturation.py --precision fp32 --out run.json
"""
from __future__ import annotations

import argparse
import json
import sys
import time
from pathlib import Path

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))

# the reference's default constants (LBM.h:34-86)
DEFAULT_CASE = dict(nx=122, ny=122, nz=101, lx=1.22, ly=1.22, nu=0.0251004, K=2.5e-5,
                    charge0=10.0, diffu=6.25e-5, lambda_f=1.0 / 12.0, lambda_g=1.0e-6)


def case_params(ehd, case: dict = DEFAULT_CASE):
    """ehd_params of a case given by the reference's own constants."""
    c = dict(case)
    eps, voltage, rho0 = 1.0e-4, 1.0e4, 1600.0
    T = eps * voltage / (c["K"] * c["nu"] * rho0)
    M = (eps / rho0) ** 0.5 / c["K"]
    C = c["charge0"] / (voltage * eps)
    Fe = c["K"] * voltage / c["diffu"]
    return ehd.params_from_groups(c["nx"], c["ny"], c["nz"], c["lx"], c["ly"], T=T, M=M, C=C,
                                  Fe=Fe, lambda_f=c["lambda_f"], lambda_g=c["lambda_g"],
                                  nu=c["nu"], K=c["K"], charge0=c["charge0"],
                                  diffu=c["diffu"])


def transit_steps(p, transits: float) -> int:
    """`transits` charge transit times Lz / (K V / Lz), an even number of steps."""
    n = int(round(transits * p.lz * p.lz / (p.K * p.voltage) / p.dt))
    return n + (n & 1)


def saturated(hist: list, tol: float, hold: int, guard: float) -> bool:
    """The criterion of the module docstring on a list of sample dicts."""
    if not any(abs(h["nu_e"] - 1.0) > guard for h in hist):
        return False
    if len(hist) < hold + 1:
        return False
    for k in range(len(hist) - hold, len(hist)):
        a, b = hist[k - 1]["nu_e"], hist[k]["nu_e"]
        if not abs(b - a) <= tol * abs(b):
            return False
    return True


def start_state(ehd, p, transits=16.0, seed=0, amp=1e-3, device=0):
    """The hydrostatic profile (FP64 column) and its I0."""
    return ehd.hydrostatic_profile(p, transit_steps(p, transits), "fp64", device)


def run(ehd, p, precision="fp32", sample_every=1000, tol=1e-3, hold=3, guard=0.01,
        max_steps=6_000_000, seed=0, amp=1e-3, transits=16.0, device=0, stream=None,
        log=None):
    import torch

    t0 = time.perf_counter()
    prof, i0 = start_state(ehd, p, transits, seed, amp, device)
    t_prof = time.perf_counter() - t0
    hist = []
    nodes = p.nx * p.ny * p.nz
    with ehd.Simulation(p, precision, device=device, stream=stream) as sim:
        sim.set_state_seeded(prof, seed=seed, amp=amp)
        sim.set_reference_current(i0)
        torch.cuda.synchronize(device)
        t1 = time.perf_counter()
        steps, status = 0, "max_steps"
        n = 2
        while steps + n <= max_steps:
            d = sim.step_sampled(n)
            steps += n
            n = sample_every
            h = {"step": steps, "nu_e": d["nu_e"], "current": d["current"],
                 "current_mean": d["current_mean"], "kinetic_energy": d["kinetic_energy"],
                 "umax": d["umax"], "total_charge": d["total_charge"]}
            hist.append(h)
            if log is not None and len(hist) % 100 == 0:
                print(json.dumps({"progress": h, "wall_s": round(time.perf_counter() - t1, 1)}),
                      file=log, flush=True)
            if d["nonfinite"]:
                status = "nonfinite"
                break
            if saturated(hist, tol, hold, guard):
                status = "saturated"
                break
        wall = time.perf_counter() - t1
    return {"precision": precision, "status": status, "steps": steps,
            "nu_e": hist[-1]["nu_e"] if hist else None, "wall_s": wall,
            "mlups": steps * nodes / wall / 1e6 if wall > 0 else None,
            "profile_wall_s": t_prof, "i0": i0, "sample_every": sample_every, "tol": tol,
            "hold": hold, "guard": guard, "seed": seed, "amp": amp, "transits": transits,
            "grid": [p.nx, p.ny, p.nz], "params": p.as_dict(), "history": hist}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--precision", default="fp32", choices=["fp64", "fp32", "mixed", "fp16", "bf16"])
    ap.add_argument("--sample-every", type=int, default=1000)
    ap.add_argument("--tol", type=float, default=1e-3)
    ap.add_argument("--hold", type=int, default=3)
    ap.add_argument("--guard", type=float, default=0.01)
    ap.add_argument("--max-steps", type=int, default=6_000_000)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--out", default=None)
    args = ap.parse_args()
    import ehd

    p = case_params(ehd)
    res = run(ehd, p, args.precision, args.sample_every, args.tol, args.hold, args.guard,
              args.max_steps, args.seed, log=sys.stderr)
    summary = {k: v for k, v in res.items() if k != "history"}
    print(json.dumps(summary), flush=True)
    if args.out:
        Path(args.out).write_text(json.dumps(res))


if __name__ == "__main__":
    main()
