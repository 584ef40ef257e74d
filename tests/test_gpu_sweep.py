"""A small T-sweep share on one GPU through sweep.run_share: every instance
runs from its hydrostatic column's state plus its seeded noise, in one batch,
and its result equals the same instance run alone with the same launch
shapes."""
import importlib.util

import pytest

from conftest import ROOT, ehd

pytestmark = pytest.mark.gpu


def load_sweep():
    spec = importlib.util.spec_from_file_location("ehd_sweep",
                                                  ROOT / "ehd-convection-3d_b200" / "sweep.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_share_runs_and_matches_lone_instances():
    S = load_sweep()
    insts = S.make_instances(4, seed=1, nz_choices=(8, 12), t_range=(200.0, 400.0))
    kw = dict(precision="fp32", sample_every=50, tol=1e-3, hold=2, max_steps=300,
              autotune=False, hydrostatic_transits=2.0)
    res = S.run_share(insts, **kw)
    assert [r["index"] for r in res] == [s["index"] for s in insts]
    for s, r in zip(insts, res):
        assert not r["nonfinite"] and 0 < r["steps"] <= 300
        p = S.instance_params(ehd, s)
        col, i0 = ehd.hydrostatic_column(p, S.hydrostatic_steps(p, 2.0))
        with ehd.Simulation(p, "fp32") as sim:  # the same instance alone
            sim.set_state_from_column(col, seed=s["seed"], amp=1e-3)
            col.close()
            sim.set_reference_current(i0)
            alone = sim.run_to_saturation(sample_every=50, tol=1e-3, hold=2, max_steps=300)
        assert (r["nu_e"], r["steps"], r["saturated"]) == (alone["nu_e"], alone["steps"],
                                                            alone["saturated"]), (s, r, alone)
