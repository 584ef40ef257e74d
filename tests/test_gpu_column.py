"""A 3D start from the hydrostatic column's own state (ehd_hydrostatic_column,
ehd_set_state_from_column): every plane then evolves as the column does, and
Nu_e stays 1 where a start from the column's fields (ehd_set_state_seeded)
perturbs the planes next to the injector."""
import numpy as np
import pytest

from conftest import ehd, relerr

pytestmark = pytest.mark.gpu


def params(nx=16, ny=12, nz=33):
    dz = 1.0 / (nz - 1)
    return ehd.params_from_groups(nx, ny, nz, nx * dz, ny * dz, T=300, M=10, C=10, Fe=4000,
                                  lambda_f=1.0 / 12.0, lambda_g=1e-6)


def transit_steps(p, transits=4.0):
    n = int(round(transits * p.lz * p.lz / (p.K * p.voltage) / p.dt))
    return n + (n & 1)


# FP32 against the FP64 column: the injector plane alternates between 2 q0
# and about 0, which FP32 resolves to about 1e-4
@pytest.mark.parametrize("prec,tol", [("fp64", 1e-11), ("fp32", 1e-4)])
def test_broadcast_column_evolves_as_the_column(prec, tol):
    p = params()
    col, i0 = ehd.hydrostatic_column(p, transit_steps(p))
    try:
        with ehd.Simulation(p, prec) as sim:
            sim.set_state_from_column(col, seed=0, amp=0.0)
            start = sim.get_fields()
            ref = col.get_fields()
            for k in ("rho", "q", "phi", "ez"):
                assert relerr(start[k], np.broadcast_to(ref[k], start[k].shape)) < tol, k
            sim.step(300)
            col.step(300)
            got, ref = sim.get_fields(), col.get_fields()
        for k in ("rho", "q", "phi", "ez"):
            assert relerr(got[k], np.broadcast_to(ref[k], got[k].shape)) < tol, (k, prec)
        assert np.abs(got["u"]).max() < 1e-9 and np.abs(got["v"]).max() < 1e-9
    finally:
        col.close()


def test_column_start_keeps_nu_e_at_one_and_the_field_start_does_not():
    p = params()
    n = transit_steps(p)
    col, i0 = ehd.hydrostatic_column(p, n)
    prof, i0p = ehd.hydrostatic_profile(p, n)
    assert i0 == pytest.approx(i0p, rel=1e-12)  # the same column, the same I0
    try:
        with ehd.Simulation(p, "fp64") as a, ehd.Simulation(p, "fp64") as b:
            a.set_state_from_column(col, amp=0.0)
            a.set_reference_current(i0)
            b.set_state_seeded(prof, amp=0.0)
            b.set_reference_current(i0)
            da = [a.step_sampled(500) for _ in range(2)]
            nu_b = [b.step_sampled(500)["nu_e"] for _ in range(2)]
            # the column itself over the same steps (its current is one node's)
            dc = [col.step_sampled(500) for _ in range(2)]
        nu_a = [d["nu_e"] for d in da]
        for x, c in zip(da, dc):
            assert x["current_mean"] == pytest.approx(c["current_mean"] * p.nx * p.ny, rel=1e-10)
        # the column is not quite converged after four transits: Nu_e drifts
        # by a few 1e-6; the start from the fields is off by a per cent
        assert all(abs(x - 1.0) < 1e-5 for x in nu_a), nu_a
        assert all(abs(x - 1.0) > 1e-3 for x in nu_b), nu_b
    finally:
        col.close()


def test_column_start_adds_the_seeded_perturbation():
    p = params()
    col, _ = ehd.hydrostatic_column(p, 2000)
    prof, _ = ehd.hydrostatic_profile(p, 2000)
    try:
        with ehd.Simulation(p, "fp32") as a, ehd.Simulation(p, "fp32") as b:
            a.set_state_from_column(col, seed=7, amp=1e-3)
            b.set_state_seeded(prof, seed=7, amp=1e-3)
            fa, fb, fc = a.get_fields(), b.get_fields(), col.get_fields()
            # the column's velocity (not yet at rest after 2000 steps) plus the
            # perturbation set_state_seeded adds to a state at rest
            for k in ("u", "v", "w"):
                assert np.abs(fa[k] - np.broadcast_to(fc[k], fa[k].shape) - fb[k]).max() < 1e-8, k
            assert np.abs(fa["u"]).max() > 5e-4
            a.step(20)
            assert not a.diagnostics()["nonfinite"]
        with ehd.Simulation(params(nz=17), "fp32") as c, pytest.raises(ehd.EhdError):
            c.set_state_from_column(col)  # another grid height
    finally:
        col.close()
