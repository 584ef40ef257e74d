"""Parity of the CUDA step (through the C ABI) with the reference and the oracle.

Tolerances (max-norm relative error per field, max|a-b|/max|b|; velocity
components relative to the largest velocity component):
  FP64 product vs the reference's own FP64 build: 1e-9 on the tiny golden
  cases (round-off only), 1e-6 after 1000 and 2000 steps of config 0 (the
  dynamics amplify round-off; the oracle itself differs by ~4e-8);
  FP32 product vs the reference on config 0: 1e-5 after 1000 steps (the bar
  of the specification), 1e-4 after 2000 steps.
"""
import numpy as np
import pytest

from conftest import O, ehd, golden, relerr

pytestmark = pytest.mark.gpu


def case(name):
    import make_golden as M
    return M, M.case_params(name)


def to_ehd(p):
    return ehd.Params.from_dict(p.as_dict())


@pytest.mark.parametrize("name", ["tiny_default", "tiny_groups"])
def test_fp64_matches_reference_golden(name):
    M, p = case(name)
    g = golden(name)
    with ehd.Simulation(to_ehd(p), "fp64") as sim:
        sim.set_fields({k: g[f"in_{k}"] for k in O.FIELDS})
        done = 0
        for n in M.CASE_STEPS[name]:
            sim.step(n - done)
            done = n
            mine = O.data_end_view(sim.get_fields())
            for k in O.FIELDS:
                e = relerr(mine[k], g[f"out{n}_{k}"])
                assert e < 1e-9, (name, n, k, e)
            cur = sim.current()
            assert cur == pytest.approx(float(g[f"current{n}"]), rel=1e-9)


def config0_inputs():
    M, p = case("config0")
    g = golden("config0")
    prof = {k: g[f"prof_{k}"] for k in O.FIELDS}
    return M, p, g, O.state_from_profile(p, prof, seed=0, amp=1e-3)


def vel_err(mine, ref, comps):
    """Error of a vector field per component relative to its largest
    component (components that vanish in exact arithmetic carry only
    round-off)."""
    scale = max(np.abs(ref[k]).max() for k in comps)
    return max(float(np.abs(mine[k] - ref[k]).max() / scale) for k in comps)


# (steps, tolerance on q, phi, velocity, E and the rho deviation)
CONFIG0_TOL = {"fp64": [(1000, 1e-8), (2000, 1e-8)],
               "fp32": [(1000, 1e-5), (2000, 1e-4)]}


def config0_errors(mine, ref, rho0):
    """Per-field errors against the reference: q, phi relative to their
    largest magnitude; velocity and E per component relative to the largest
    component of the vector; rho relative to 1600 and, for FP64, its deviation
    from rho0 relative to the largest deviation."""
    err = {"q": relerr(mine["q"], ref["q"]), "phi": relerr(mine["phi"], ref["phi"]),
           "velocity": vel_err(mine, ref, ("u", "v", "w")),
           "E": vel_err(mine, ref, ("ex", "ey", "ez")), "rho": relerr(mine["rho"], ref["rho"])}
    dev = np.abs(ref["rho"] - rho0).max()
    err["rho_dev"] = float(np.abs(mine["rho"] - ref["rho"]).max() / dev)
    return err


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_config0_matches_reference(prec):
    """64 x 64 x 33, hydrostatic start + seeded 1e-3 noise: all nine fields and
    the collector current after 1000 and 2000 steps against the reference's own
    build (FP64 fixtures, fields as its data_end.dat writer reports them)."""
    M, p, g, f = config0_inputs()
    with ehd.Simulation(to_ehd(p), prec) as sim:
        sim.set_fields(f)
        done = 0
        for n, tol in CONFIG0_TOL[prec]:
            sim.step(n - done)
            done = n
            mine = O.data_end_view(sim.get_fields())
            ref = {k: g[f"out{n}_{k}"] for k in O.FIELDS}
            err = config0_errors(mine, ref, p.rho0)
            for k in ("q", "phi", "velocity", "E"):
                assert err[k] < tol, (prec, n, k, err)
            if prec == "fp64":
                assert err["rho_dev"] < tol, (prec, n, err)
            else:  # FP32 rho: 1600 plus deviations of a few units
                assert err["rho"] < 1e-6, (prec, n, err)
            assert sim.current() == pytest.approx(float(g[f"current{n}"]), rel=tol)


def test_config0_mixed_storage_matches_reference():
    """Mixed storage (FP16 deviations of the flow populations, FP32 of the
    charge populations) on config 0 against the reference's own build after
    1000 steps.  The charge keeps FP32 storage, so q and phi stay near FP32
    accuracy; the velocity and rho carry the FP16 rounding of f.  Tolerances:
    q 5e-4, phi 1e-5, E 1e-4, velocity 5e-3 (per component of the vector), rho
    2e-5 relative to 1600 (measured 2.3e-4, 1.6e-6, 1.2e-5, 8.7e-4, 6.0e-6)."""
    M, p, g, f = config0_inputs()
    with ehd.Simulation(to_ehd(p), "mixed") as sim:
        sim.set_fields(f)
        sim.step(1000)
        mine = O.data_end_view(sim.get_fields())
    ref = {k: g[f"out1000_{k}"] for k in O.FIELDS}
    err = config0_errors(mine, ref, p.rho0)
    for k, tol in (("q", 5e-4), ("phi", 1e-5), ("E", 1e-4), ("velocity", 5e-3), ("rho", 2e-5)):
        assert err[k] < tol, (k, err)


def random_fields(p, seed):
    import make_golden as M
    return M.random_fields(p, seed)


@pytest.mark.parametrize("shape", [(16, 12, 9), (48, 20, 11), (30, 25, 7), (1, 1, 17),
                                   (22, 14, 9), (122, 122, 101)])
def test_step_halves_match_oracle(shape):
    """The LBM half (stream_collide_save) and the Poisson half, separately and
    then chained, against the oracle on grids with radix 2, 3 and 5 factors,
    other primes (22 = 2 x 11, 14 = 2 x 7), and the reference's own default
    grid 122 x 122 x 101 (LBM.h:34-36: 122 = 2 x 61, Thomas z solve)."""
    nx, ny, nz = shape
    dz = 1.0 / (nz - 1)
    p = O.params_from_groups(nx, ny, nz, nx * dz, ny * dz, T=200, M=10, C=10, Fe=4000,
                             exf=50.0, uw=0.01)
    f = random_fields(p, 21)
    o = O.Oracle(p)
    o.set_fields(f)
    with ehd.Simulation(to_ehd(p), "fp64") as sim:
        sim.set_fields(f)
        sim.stream_collide_save()
        o.step_lbm()
        a, b = sim.get_fields(), o.get_fields()
        for k in ("rho", "u", "v", "w", "q"):
            assert relerr(a[k], b[k]) < 1e-12, ("lbm", k)
        for k in ("phi", "ex", "ey", "ez"):
            assert np.array_equal(a[k], f[k]), k  # unchanged until the Poisson solve
        sim.poisson()
        o.poisson()
        o.efield()
        a, b = sim.get_fields(), o.get_fields()
        # the z operator's condition number grows as NZ^2 (the FP64 solve of
        # NZ = 101 loses a decade more than the small grids)
        tol_p = 1e-11 * max(1.0, (nz / 33.0) ** 2)
        for k in ("phi", "ex", "ey", "ez"):
            assert relerr(a[k], b[k]) < tol_p, ("poisson", k, relerr(a[k], b[k]))
        sim.step(5)
        o.step(5)
        a, b = sim.get_fields(), o.get_fields()
        for k in O.FIELDS:
            assert relerr(a[k], b[k]) < 1e-10, ("step", k, relerr(a[k], b[k]))


@pytest.mark.parametrize("shape", [(256, 128, 9), (128, 256, 7), (512, 64, 5), (64, 512, 5),
                                   (256, 96, 6), (122, 122, 7), (14, 77, 5), (61, 26, 6),
                                   (127, 13, 5), (96, 96, 49), (80, 48, 41), (48, 80, 25)])
@pytest.mark.parametrize("prec,tol", [("fp64", 1e-11), ("fp32", 2e-6)])
def test_poisson_fft_sizes_match_oracle(shape, prec, tol):
    """The compile-time-radix FFT paths (N = 48, 64, 80, 96, 128, 256, 512, two
    real rows per transform; the z sine transforms of length 48, 80, 96 on the
    T-sweep grids) and the run-time radix path (radix 2/3/4/5 and the direct
    radix-p passes for other primes: 122 = 2 x 61, the reference's own grid
    width, LBM.h:34-35; 77 = 7 x 11; prime and odd widths), against the
    oracle's odd-extension DFT solve (poisson.cu:78-167) on random charge."""
    nx, ny, nz = shape
    dz = 1.0 / (nz - 1)
    p = O.params_from_groups(nx, ny, nz, nx * dz, ny * dz, T=200, M=10, C=10, Fe=4000)
    f = random_fields(p, 3)
    o = O.Oracle(p)
    o.set_fields(f)
    o.poisson()
    o.efield()
    b = o.get_fields()
    with ehd.Simulation(to_ehd(p), prec) as sim:
        sim.set_fields(f)
        sim.poisson()
        a = sim.get_fields()
    for k in ("phi", "ex", "ey", "ez"):
        assert relerr(a[k], b[k]) < tol, (k, relerr(a[k], b[k]))


@pytest.mark.parametrize("shape", [(256, 256, 129), (64, 64, 33), (128, 256, 65), (512, 64, 17),
                                   (64, 512, 33), (256, 128, 129), (128, 128, 257)])
@pytest.mark.parametrize("prec,tol", [("fp64", 1e-10), ("fp32", 2e-6)])
def test_poisson_split_path_matches_oracle_and_five_kernel_path(shape, prec, tol):
    """The three-kernel split-y Poisson solve (the x-row kernels fold in the
    radix-S first and last stages of the y transform, NY = 64 S; one slab
    kernel per (kx, j) runs the 64-point y transforms and the Thomas z solve
    in FP64 arithmetic on chip) against the oracle's odd-extension DFT solve
    (poisson.cu:78-167) and against the five-kernel path of the same context
    type (ehd_tuning.poisson_path = 1), on random charge."""
    nx, ny, nz = shape
    dz = 1.0 / (nz - 1)
    p = O.params_from_groups(nx, ny, nz, nx * dz, ny * dz, T=200, M=10, C=10, Fe=4000)
    f = random_fields(p, 5)
    o = O.Oracle(p)
    o.set_fields(f)
    o.poisson()
    o.efield()
    b = o.get_fields()
    o.close()
    out = {}
    for path in (0, 1):
        with ehd.Simulation(to_ehd(p), prec) as sim:
            sim.set_tuning(poisson_path=path)
            sim.set_fields(f)
            sim.poisson()
            out[path] = sim.get_fields()
    for k in ("phi", "ex", "ey", "ez"):
        assert relerr(out[0][k], b[k]) < tol, (k, "oracle", relerr(out[0][k], b[k]))
        assert relerr(out[0][k], out[1][k]) < tol, (k, "five-kernel", relerr(out[0][k], out[1][k]))


@pytest.mark.parametrize("shape", [(96, 96, 49), (80, 80, 41), (48, 48, 25), (64, 96, 65),
                                   (122, 80, 33)])
@pytest.mark.parametrize("prec,tol", [("fp64", 1e-10), ("fp32", 2e-6)])
def test_fused_yz_path_matches_oracle_and_five_kernel_path(shape, prec, tol):
    """For NY = 48, 80 or 96 (the T-sweep grids, which the split-y path does
    not take) and L = 2 (NZ - 1) a compile-time size, one kernel does the y
    transform, the sine-transform z solve and the inverse y transform of
    every kx column block (poisson_yz); against the oracle's odd-extension DFT
    solve (poisson.cu:78-167) and the five-kernel path (ehd_tuning.poisson_path
    = 1) on random charge, with a run-time-radix x transform in the last case
    (122 = 2 x 61)."""
    nx, ny, nz = shape
    dz = 1.0 / (nz - 1)
    p = O.params_from_groups(nx, ny, nz, nx * dz, ny * dz, T=200, M=10, C=10, Fe=4000)
    f = random_fields(p, 6)
    o = O.Oracle(p)
    o.set_fields(f)
    o.poisson()
    o.efield()
    b = o.get_fields()
    o.close()
    out = {}
    for path in (0, 1):
        with ehd.Simulation(to_ehd(p), prec) as sim:
            sim.set_tuning(poisson_path=path)
            sim.set_fields(f)
            sim.poisson()
            out[path] = sim.get_fields()
    for k in ("phi", "ex", "ey", "ez"):
        assert relerr(out[0][k], b[k]) < tol, (k, "oracle", relerr(out[0][k], b[k]))
        assert relerr(out[0][k], out[1][k]) < tol, (k, "five-kernel", relerr(out[0][k], out[1][k]))


@pytest.mark.parametrize("shape", [(48, 40, 27), (122, 122, 101), (30, 25, 7)])
@pytest.mark.parametrize("prec,tol", [("fp64", 1e-10), ("fp32", 2e-6)])
def test_z_solve_choices_match_oracle(shape, prec, tol):
    """Where 2 (NZ - 1) is not a compile-time FFT size, the z solve is the sine
    transform with run-time FFT passes (ehd_tuning.z_solve = 0) or the FP64
    Thomas sweep (z_solve = 1); both against the oracle's odd-extension DFT
    solve (poisson.cu:78-167) on random charge."""
    nx, ny, nz = shape
    dz = 1.0 / (nz - 1)
    p = O.params_from_groups(nx, ny, nz, nx * dz, ny * dz, T=200, M=10, C=10, Fe=4000)
    f = random_fields(p, 6)
    o = O.Oracle(p)
    o.set_fields(f)
    o.poisson()
    o.efield()
    b = o.get_fields()
    o.close()
    for zs in (0, 1):
        with ehd.Simulation(to_ehd(p), prec) as sim:
            sim.set_tuning(z_solve=zs)
            sim.set_fields(f)
            sim.poisson()
            a = sim.get_fields()
        for k in ("phi", "ex", "ey", "ez"):
            assert relerr(a[k], b[k]) < tol, (zs, k, relerr(a[k], b[k]))


@pytest.mark.parametrize("shape", [(64, 48, 33), (96, 64, 65), (32, 20, 129), (16, 12, 257)])
@pytest.mark.parametrize("prec,tol", [("fp64", 1e-10), ("fp32", 2e-6)])
def test_poisson_sine_transform_z_solve_matches_oracle(shape, prec, tol):
    """2 (NZ - 1) = 64..512: the z solve runs as a sine transform (odd
    extension, FFT, spectral division, FFT) instead of the Thomas sweep;
    against the oracle's odd-extension DFT solve on random charge.  The z
    operator's condition number grows as NZ^2 (about 3e4 at NZ = 257), which
    sets the FP64 tolerance."""
    nx, ny, nz = shape
    dz = 1.0 / (nz - 1)
    p = O.params_from_groups(nx, ny, nz, nx * dz, ny * dz, T=200, M=10, C=10, Fe=4000)
    f = random_fields(p, 4)
    o = O.Oracle(p)
    o.set_fields(f)
    o.poisson()
    o.efield()
    b = o.get_fields()
    with ehd.Simulation(to_ehd(p), prec) as sim:
        sim.set_fields(f)
        sim.poisson()
        a = sim.get_fields()
    for k in ("phi", "ex", "ey", "ez"):
        assert relerr(a[k], b[k]) < tol, (k, relerr(a[k], b[k]))


def test_graphs_and_direct_launches_agree_bitwise():
    _, p, _, f = config0_inputs()
    out = []
    for graphs in (True, False):
        with ehd.Simulation(to_ehd(p), "fp32", graphs=graphs) as sim:
            sim.set_fields(f)
            sim.step(7)
            sim.step(6)
            out.append(sim.get_fields())
    for k in O.FIELDS:
        assert np.array_equal(out[0][k], out[1][k]), k


def test_runs_are_deterministic():
    _, p, _, f = config0_inputs()
    res = []
    for _ in range(2):
        with ehd.Simulation(to_ehd(p), "fp32") as sim:
            sim.set_fields(f)
            sim.step(50)
            res.append((sim.get_fields(), sim.diagnostics()))
    for k in O.FIELDS:
        assert np.array_equal(res[0][0][k], res[1][0][k]), k
    assert res[0][1] == res[1][1]


def test_reference_initialization_matches_oracle():
    """ehd_initialize = initialization + init_equilibrium (LBM.cu:69-276)."""
    p = O.params_from_groups(16, 16, 9, 2.0, 2.0, T=200, M=10, C=10, Fe=4000)
    o = O.Oracle(p)
    o.initialization()
    with ehd.Simulation(to_ehd(p), "fp64") as sim:
        sim.initialize()
        a = sim.get_fields()
        b = o.get_fields()
        for k in O.FIELDS:
            np.testing.assert_array_equal(a[k], b[k])
        sim.step(20)
        o.step(20)
        a, b = sim.get_fields(), o.get_fields()
        for k in ("rho", "q", "phi"):
            assert relerr(a[k], b[k]) < 1e-10, k
        assert vel_err(a, b, ("u", "v", "w")) < 1e-10
        assert vel_err(a, b, ("ex", "ey", "ez")) < 1e-10


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_diagnostics_match_host_reductions(prec):
    _, p, _, f = config0_inputs()
    with ehd.Simulation(to_ehd(p), prec) as sim:
        sim.set_fields(f)
        sim.step(30)
        d = sim.diagnostics()
        cur = sim.current()  # the collector plane alone, another summation order
        fl = sim.get_fields()
    dv = p.dx * p.dy * p.dz
    rtol = 1e-12 if prec == "fp64" else 1e-6
    assert d["current"] == pytest.approx(O.current_of(p, fl["q"], fl["ez"]), rel=rtol)
    assert cur == pytest.approx(d["current"], rel=1e-13)
    ke = 0.5 * np.sum(fl["rho"] * (fl["u"] ** 2 + fl["v"] ** 2 + fl["w"] ** 2)) * dv
    assert d["kinetic_energy"] == pytest.approx(ke, rel=rtol)
    assert d["total_charge"] == pytest.approx(np.sum(fl["q"]) * dv, rel=rtol)
    w = fl["w"].copy()
    w[-1] = 2 * w[-2] - w[-3]
    assert d["umax"] == pytest.approx(max(0.0, w.max()), rel=rtol)
    assert d["step"] == 30 and d["nonfinite"] == 0
    assert d["time"] == pytest.approx(30 * p.dt)


@pytest.mark.parametrize("prec", ["fp16", "bf16"])
def test_reduced_storage_runs_and_stays_close(prec):
    """FP16/BF16 population storage: finite, and close to FP64 over 200 steps
    (longer runs are compared field by field by precision.py)."""
    _, p, _, f = config0_inputs()
    res = {}
    for pr in ("fp64", prec):
        with ehd.Simulation(to_ehd(p), pr) as sim:
            sim.set_fields(f)
            sim.step(200)
            res[pr] = sim.get_fields()
            assert sim.diagnostics()["nonfinite"] == 0
    for k in ("q", "phi", "rho"):
        assert relerr(res[prec][k], res["fp64"][k]) < 5e-2, k
