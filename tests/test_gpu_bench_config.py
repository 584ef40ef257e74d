"""Parity at the benchmark's own configuration: 256 x 256 x 129 nodes,
Lx = Ly = 2, T = 200, M = 10, C = 10, Fe = 4000, TRT 1/4, FP32 populations,
the reference's initial state plus the seeded 1e-3 velocity noise
(bench.workload_params, bench.initial_fields).  Every performance figure of
bench.py comes from this case: the first step on the per-node kernel, every
later step on the bulk-copy row kernel at NX = 256 and the sine-transform z
solve of length 256.

Tolerances (max-norm relative error per field; velocity and E per component
relative to the largest component of the vector):
  FP32 against the oracle (FP64) after 1 and 5 steps: 1e-5 (the bar for FP32
  fields), velocity and E 1e-5;
  FP32 against the product's own FP64 run after 1000 steps: 1e-5 on q and phi,
  1e-4 on velocity and E, 1e-6 on rho (1600 plus deviations that the FP32
  field resolves to about 1e-4).
"""
import importlib.util
import os

import numpy as np
import pytest

from conftest import O, ROOT, ehd, relerr

pytestmark = pytest.mark.gpu


def bench_module():
    spec = importlib.util.spec_from_file_location("bench_for_tests", ROOT / "bench.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def vec_err(mine, ref, comps):
    scale = max(float(np.abs(ref[k]).max()) for k in comps)
    if scale == 0.0:
        scale = 1.0
    return max(float(np.abs(mine[k] - ref[k]).max()) / scale for k in comps)


def field_errors(mine, ref):
    out = {k: relerr(mine[k], ref[k]) for k in ("rho", "q", "phi")}
    out["velocity"] = vec_err(mine, ref, ("u", "v", "w"))
    out["E"] = vec_err(mine, ref, ("ex", "ey", "ez"))
    return out


@pytest.fixture(scope="module")
def case():
    B = bench_module()
    p = B.workload_params(ehd)
    assert (p.nx, p.ny, p.nz) == (256, 256, 129)
    return B, p, B.initial_fields(p, seed=0)


def test_bench_case_fp32_matches_oracle_after_1_and_5_steps(case):
    B, p, f = case
    O.set_threads(os.cpu_count() or 1)
    o = O.Oracle(O.Params(**p.as_dict()))
    o.set_fields(f)
    with ehd.Simulation(p, "fp32") as sim:
        sim.set_fields(f)
        tun = sim.get_tuning()
        assert tun["lbm_kernel"] == 0  # the row kernel serves the steady steps
        done = 0
        for n in (1, 5):
            sim.step(n - done)
            o.step(n - done)
            done = n
            err = field_errors(sim.get_fields(), o.get_fields())
            for k, e in err.items():
                assert e < 1e-5, (n, k, err)
    o.close()


def test_bench_case_fp32_matches_fp64_after_1000_steps(case):
    B, p, f = case
    res = {}
    for prec in ("fp64", "fp32"):
        with ehd.Simulation(p, prec) as sim:
            sim.set_fields(f)
            sim.step(1000)
            res[prec] = sim.get_fields()
            assert sim.diagnostics()["nonfinite"] == 0
    a, b = res["fp32"], res["fp64"]
    err = field_errors(a, b)
    for k in ("q", "phi"):
        assert err[k] < 1e-5, (k, err)
    for k in ("velocity", "E"):
        assert err[k] < 1e-4, (k, err)
    # rho is 1600 plus deviations of a few tenths: the FP32 field resolves it
    # to about 1e-4 absolute
    assert err["rho"] < 1e-6, err
