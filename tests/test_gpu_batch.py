"""Batches of independent instances (ehd_batch): one graph launch per step over
every active instance, per-instance run to saturation, and the autotuner.

Mode 1 (a graph branch per instance, the default): an instance runs the same
kernels with the same launch shapes as a lone context, checked bitwise.
Mode 0 (grouped launches): each kernel of a step is one launch over every
instance with the same grid, the LBM half on the per-node kernel; the grouped
kernels are separate compilations, whose multiply-add contractions may differ
from the lone kernels', so mode 0 is checked against lone contexts on the
per-node kernel to FP32 round-off.
"""
import numpy as np
import pytest

from conftest import O, ehd, relerr

pytestmark = pytest.mark.gpu

# uneven grids: row kernel (64 wide), per-node kernel with run-time-radix FFTs
# (48 and 80 wide), odd NZ for the Thomas z solve (25) and the sine transform (33)
SHAPES = [(64, 64, 33), (48, 48, 25), (80, 40, 17)]


def params(shape, T=200.0):
    nx, ny, nz = shape
    dz = 1.0 / (nz - 1)
    return O.params_from_groups(nx, ny, nz, nx * dz, ny * dz, T=T, M=10, C=10, Fe=4000)


def to_ehd(p):
    return ehd.Params.from_dict(p.as_dict())


def fields(p, seed):
    import make_golden as M
    return M.random_fields(p, seed)


@pytest.mark.parametrize("mode", [0, 1])
def test_batch_steps_match_lone_contexts(mode):
    ps = [params(s, T) for s, T in zip(SHAPES, (150.0, 250.0, 350.0))]
    # a fourth instance on the first grid: a group of two in mode 0
    ps.append(params(SHAPES[0], 300.0))
    fs = [fields(p, 30 + i) for i, p in enumerate(ps)]
    lone = []
    for p, f in zip(ps, fs):
        with ehd.Simulation(to_ehd(p), "fp32", row_kernel=mode == 1) as sim:
            sim.set_fields(f)
            sim.step(4)
            sim.step(6)
            lone.append((sim.get_fields(), sim.diagnostics()))
    with ehd.Batch([to_ehd(p) for p in ps], "fp32") as b:
        b.set_mode(mode)
        for sim, f in zip(b, fs):
            sim.set_fields(f)
        b.step(4)
        b.step(6)
        for i, sim in enumerate(b):
            out, d = sim.get_fields(), sim.diagnostics()
            for k in O.FIELDS:
                if mode == 1:
                    assert np.array_equal(out[k], lone[i][0][k]), (i, k)
                else:
                    assert relerr(out[k], lone[i][0][k]) < 1e-5, (i, k, relerr(out[k], lone[i][0][k]))
            if mode == 1:
                assert d == lone[i][1]


def test_grouped_launches_keep_each_instances_voltage_and_permittivity():
    """Mode 0 groups instances only where a grouped Poisson launch may take
    its constants from the group's first member: three instances on one grid
    that differ in electrode voltage or permittivity (both enter the Poisson
    right-hand side, poisson.cu:87-117) each match a lone context."""
    base = params(SHAPES[0], 200.0).as_dict()
    ds = [base, dict(base, voltage=1.5 * base["voltage"]), dict(base, eps=2.0 * base["eps"])]
    p0 = params(SHAPES[0], 200.0)
    fs = [fields(p0, 50 + i) for i in range(len(ds))]
    lone = []
    for d, f in zip(ds, fs):
        with ehd.Simulation(ehd.Params.from_dict(d), "fp32", row_kernel=False) as sim:
            sim.set_fields(f)
            sim.step(5)
            lone.append(sim.get_fields())
    with ehd.Batch([ehd.Params.from_dict(d) for d in ds], "fp32") as b:
        b.set_mode(0)
        for sim, f in zip(b, fs):
            sim.set_fields(f)
        b.step(5)
        for i, sim in enumerate(b):
            out = sim.get_fields()
            for k in O.FIELDS:
                assert relerr(out[k], lone[i][k]) < 1e-5, (i, k, relerr(out[k], lone[i][k]))


def test_batch_inactive_instances_do_not_advance():
    ps = [params(s) for s in SHAPES[:2]]
    with ehd.Batch([to_ehd(p) for p in ps], "fp32") as b:
        for i, sim in enumerate(b):
            sim.set_fields(fields(ps[i], 40 + i))
        b.step(3)
        before = b[1].get_fields()
        b.set_active(1, False)
        b.step(5)
        assert b[0].diagnostics()["step"] == 8
        assert b[1].diagnostics()["step"] == 3
        after = b[1].get_fields()
        for k in O.FIELDS:
            assert np.array_equal(before[k], after[k]), k
        b.set_active(1, True)
        b.step(2)
        assert b[1].diagnostics()["step"] == 5


@pytest.mark.parametrize("mode", [1])
def test_batch_run_to_saturation_matches_lone_runs(mode):
    """Each instance stops on its own: the same sampling and stopping as
    ehd_run_to_saturation on a lone context, instance by instance."""
    ps = [params(s, T) for s, T in zip(SHAPES, (150.0, 250.0, 350.0))]
    starts = []
    for p in ps:
        prof, i0 = ehd.hydrostatic_profile(to_ehd(p), 2000)
        starts.append((prof, i0))
    # tolerances that stop the instances after different numbers of samples
    lone = []
    for (prof, i0), p in zip(starts, ps):
        with ehd.Simulation(to_ehd(p), "fp32", row_kernel=mode == 1) as sim:
            sim.set_state_seeded(prof, seed=3, amp=1e-3)
            sim.set_reference_current(i0)
            lone.append(sim.run_to_saturation(sample_every=20, tol=2e-2, hold=2, max_steps=200))
    with ehd.Batch([to_ehd(p) for p in ps], "fp32") as b:
        b.set_mode(mode)
        for sim, (prof, i0) in zip(b, starts):
            sim.set_state_seeded(prof, seed=3, amp=1e-3)
            sim.set_reference_current(i0)
        res = b.run_to_saturation(sample_every=20, tol=2e-2, hold=2, max_steps=200)
    for i, (r, l) in enumerate(zip(res, lone)):
        assert r["steps"] == l["steps"] and r["saturated"] == l["saturated"], (i, r, l)
        assert r["nu_e"] == l["nu_e"], (i, r, l)


def test_batch_run_to_saturation_needs_reference_current():
    ps = [params(s) for s in SHAPES[:2]]
    with ehd.Batch([to_ehd(p) for p in ps], "fp32") as b:
        for i, sim in enumerate(b):
            sim.set_fields(fields(ps[i], 50 + i))
        with pytest.raises(ehd.EhdError):
            b.run_to_saturation(sample_every=10, max_steps=20)


def test_autotune_picks_allowed_shapes_and_keeps_parity():
    ps = [params(s) for s in SHAPES] + [params(SHAPES[1], 300.0)]
    fs = [fields(p, 60 + i) for i, p in enumerate(ps)]
    refs = []
    for p, f in zip(ps, fs):
        o = O.Oracle(p)
        o.set_fields(f)
        o.step(6)
        refs.append(o.get_fields())
    with ehd.Batch([to_ehd(p) for p in ps], "fp32") as b:
        b.autotune(trial_steps=5)
        tunes = [sim.get_tuning() for sim in b]
        for t in tunes:
            assert t["lbm_kernel"] in (0, 1) and t["node_block_x"] in (16, 32, 64, 128)
            assert t["fft_rows"] >= 1 and t["fft_cols"] >= 1
        assert tunes[1] == tunes[3]  # one choice per distinct grid
        for sim, f in zip(b, fs):
            sim.set_fields(f)
        b.step(6)
        for i, sim in enumerate(b):
            out = sim.get_fields()
            for k in ("q", "phi", "rho"):
                assert relerr(out[k], refs[i][k]) < 1e-5, (i, k, relerr(out[k], refs[i][k]))
