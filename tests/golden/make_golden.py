"""Generate the golden vectors that pin the oracle to the reference.

The reference has no tests or fixtures of its own.  Its own CUDA build
(compiled by oracle/build_ref.py into oracle/_ref/<case>/ehd_ref) is run on a
B200 through its restart path: the seeded initial fields go in through
data_end.dat (read_data, LBM.cu:1597-1622, which rebuilds equilibrium
populations), the time loop runs EHD_REF_NSTEPS steps, and the fields come
back out of data_end.dat (save_data_end, LBM.cu:1506-1566, patched to %.17g).

Usage
  on a GPU machine:   python tests/golden/make_golden.py run  OUTDIR
  here afterwards:    python tests/golden/make_golden.py collect OUTDIR

`run` writes raw per-run .npz files to OUTDIR; `collect` packs them into the
committed fixtures tests/golden/<case>.npz.  Each case is run twice to record
the reference's run-to-run spread (its z=0 / z=1 read-write race).
"""
from __future__ import annotations

import json
import os
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT / "oracle"))
import oracle as O  # noqa: E402

GOLDEN = Path(__file__).resolve().parent
REF = ROOT / "oracle" / "_ref"
COLS = ("t", "u", "v", "w", "rho", "q", "phi", "ex", "ey", "ez")  # LBM.cu:1551-1553

CASE_STEPS = {
    "tiny_default": [1, 10, 100],
    "tiny_groups": [1, 10, 100],
    "config0": [1000, 2000],
}


def case_params(name: str) -> O.Params:
    if name == "tiny_default":
        return O.reference_default_params(16, 16, 9)
    if name == "tiny_groups":
        d = 1.0 / 12
        return O.params_from_groups(24, 16, 13, 24 * d, 16 * d, T=200, M=10, C=10, Fe=4000,
                                    uw=0.05, exf=100.0)
    if name == "config0":
        return O.params_from_groups(64, 64, 33, 2.0, 2.0, T=200, M=10, C=10, Fe=4000)
    raise KeyError(name)


def random_fields(p: O.Params, seed: int) -> dict:
    """Seeded, deliberately non-equilibrium fields that exercise every term."""
    rng = np.random.default_rng(seed)
    sh = (p.nz, p.ny, p.nx)
    r = lambda: 2.0 * rng.random(sh) - 1.0  # noqa: E731
    z = np.arange(p.nz)[:, None, None] * p.dz
    return dict(rho=p.rho0 * (1.0 + 0.01 * r()), u=0.05 * r(), v=0.05 * r(), w=0.05 * r(),
                q=10.0 * rng.random(sh), phi=p.voltage * (1.0 - z / p.lz) + 10.0 * r(),
                ex=1.0e3 * r(), ey=1.0e3 * r(), ez=1.0e4 + 1.0e3 * r())


def hydrostatic_steps(p: O.Params) -> int:
    """16 charge transit times Lz / (K V / Lz), rounded to an even count."""
    n = int(round(16.0 * p.lz * p.lz / (p.K * p.voltage) / p.dt))
    return n + (n & 1)


def case_inputs(name: str, p: O.Params):
    if name == "tiny_default":
        return random_fields(p, 1234), {}
    if name == "tiny_groups":
        return random_fields(p, 5678), {}
    nthr = O.get_threads()
    O.set_threads(1)
    prof, steps = O.hydrostatic_profile(p, tol=-1.0, check_every=hydrostatic_steps(p),
                                        max_steps=hydrostatic_steps(p))
    O.set_threads(nthr)
    prof = dict(prof)
    prof["u"][:] = 0.0
    prof["v"][:] = 0.0
    prof["w"][:] = 0.0
    f = O.state_from_profile(p, prof, seed=0, amp=1.0e-3)
    return f, {"profile": prof, "profile_steps": steps, "seed": 0, "amp": 1.0e-3}


def write_data_end(path: Path, f: dict) -> None:
    cols = [np.zeros(f["rho"].size)] + [f[k].ravel() for k in COLS[1:]]
    np.savetxt(path, np.stack(cols, axis=1), fmt="%.17g")


def read_data_end(path: Path, p: O.Params) -> dict:
    a = np.loadtxt(path)
    sh = (p.nz, p.ny, p.nx)
    return {k: a[:, i].reshape(sh) for i, k in enumerate(COLS) if k != "t"}


def run(outdir: Path) -> None:
    outdir.mkdir(parents=True, exist_ok=True)
    for name, steps in CASE_STEPS.items():
        p = case_params(name)
        f, meta = case_inputs(name, p)
        exe = REF / name / "ehd_ref"
        np.savez_compressed(outdir / f"{name}_inputs.npz",
                            params=json.dumps(p.as_dict()), meta=json.dumps(
                                {k: v for k, v in meta.items() if k != "profile"}),
                            **{f"in_{k}": v for k, v in f.items()},
                            **{f"prof_{k}": v for k, v in meta.get("profile", {}).items()})
        for n in steps:
            for rep in range(2):
                with tempfile.TemporaryDirectory() as tmp:
                    tmp = Path(tmp)
                    write_data_end(tmp / "data_end.dat", f)
                    t0 = time.time()
                    r = subprocess.run([str(exe)], cwd=tmp, capture_output=True, text=True,
                                       env=dict(os.environ, EHD_REF_NSTEPS=str(n)),
                                       timeout=600)
                    if r.returncode != 0:
                        raise RuntimeError(f"{name} n={n}: rc={r.returncode}\n{r.stdout[-2000:]}"
                                           f"\n{r.stderr[-2000:]}")
                    out = read_data_end(tmp / "data_end.dat", p)
                    np.savez_compressed(outdir / f"{name}_{n}_{rep}.npz", **out,
                                        stdout=r.stdout[-3000:], wall=time.time() - t0)
                    print(f"{name} steps={n} rep={rep} wall={time.time() - t0:.1f}s", flush=True)


def collect(indir: Path) -> None:
    for name, steps in CASE_STEPS.items():
        inp = np.load(indir / f"{name}_inputs.npz")
        p = case_params(name)
        pack = {"params": inp["params"], "meta": inp["meta"]}
        if name == "config0":
            for k in O.FIELDS:
                pack[f"prof_{k}"] = inp[f"prof_{k}"]
        else:
            for k in O.FIELDS:
                pack[f"in_{k}"] = inp[f"in_{k}"]
        for n in steps:
            a = np.load(indir / f"{name}_{n}_0.npz")
            b = np.load(indir / f"{name}_{n}_1.npz")
            # every field in FP64 (the reference's data_end.dat, %.17g)
            for k in O.FIELDS:
                pack[f"out{n}_{k}"] = a[k].astype(np.float64)
                scale = max(np.abs(a[k]).max(), 1e-300)
                pack[f"spread{n}_{k}"] = np.float64(np.abs(a[k] - b[k]).max() / scale)
            pack[f"current{n}"] = np.float64(O.current_of(p, a["q"], a["ez"]))
        np.savez_compressed(GOLDEN / f"{name}.npz", **pack)
        print("wrote", GOLDEN / f"{name}.npz", (GOLDEN / f"{name}.npz").stat().st_size)


if __name__ == "__main__":
    mode, d = sys.argv[1], Path(sys.argv[2])
    {"run": run, "collect": collect}[mode](d)
