"""The oracle against the reference's golden vectors and against the math.

CPU only.  The golden vectors come from the reference's own CUDA build run on
a B200 (tests/golden/make_golden.py); the known-answer tests follow the
reference's formulas (LBM.cu, poisson.cu) directly.
"""
import numpy as np
import pytest

from conftest import O, golden, relerr

EV = np.array([[0, 0, 0], [1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1],
               [1, 1, 0], [-1, -1, 0], [1, 0, 1], [-1, 0, -1], [0, 1, 1], [0, -1, -1],
               [1, -1, 0], [-1, 1, 0], [1, 0, -1], [-1, 0, 1], [0, 1, -1], [0, -1, 1],
               [1, 1, 1], [-1, -1, -1], [1, 1, -1], [-1, -1, 1], [1, -1, 1], [-1, 1, -1],
               [-1, 1, 1], [1, -1, -1]])
W = np.array([8 / 27] + [2 / 27] * 6 + [1 / 54] * 12 + [1 / 216] * 8)


def opp(d):
    return d + 1 if d % 2 else d - 1


@pytest.mark.parametrize("n", [1, 2, 3, 5, 8, 12, 30, 48, 64, 80, 96, 100, 128, 256, 7, 13])
def test_fft_matches_numpy(n):
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    np.testing.assert_allclose(O.fft1d(x, -1), np.fft.fft(x), atol=1e-12 * n, rtol=0)
    np.testing.assert_allclose(O.fft1d(x, +1), np.fft.ifft(x) * n, atol=1e-12 * n, rtol=0)


@pytest.mark.parametrize("case", ["tiny_default", "tiny_groups"])
def test_oracle_matches_reference_golden(case):
    """The oracle reproduces the reference's own step, all nine fields, after
    1, 10 and 100 steps from seeded non-equilibrium fields."""
    import make_golden as M
    g = golden(case)
    p = M.case_params(case)
    o = O.Oracle(p)
    o.set_fields({k: g[f"in_{k}"] for k in O.FIELDS})
    done = 0
    for n in M.CASE_STEPS[case]:
        o.step(n - done)
        done = n
        mine = O.data_end_view(o.get_fields())
        for k in O.FIELDS:
            ref = g[f"out{n}_{k}"]
            assert float(g[f"spread{n}_{k}"]) == 0.0  # reference run-to-run spread
            assert relerr(mine[k], ref) < 1e-11, (case, n, k, relerr(mine[k], ref))
        assert abs(o.current() - float(g[f"current{n}"])) <= 1e-11 * abs(float(g[f"current{n}"]))


def test_oracle_matches_reference_config0_1000_steps():
    """The oracle against the reference's own build on config 0 (64 x 64 x 33,
    hydrostatic start + seeded noise, FP64 fixtures from its data_end.dat):
    every field after 1000 steps; velocity and E per component relative to
    the largest component of the vector, rho as its deviation from rho0."""
    import make_golden as M
    g = golden("config0")
    p = M.case_params("config0")
    prof = {k: g[f"prof_{k}"] for k in O.FIELDS}
    o = O.Oracle(p)
    o.set_fields(O.state_from_profile(p, prof, seed=0, amp=1e-3))
    o.step(1000)
    mine = O.data_end_view(o.get_fields())
    o.close()
    ref = {k: g[f"out1000_{k}"] for k in O.FIELDS}

    def vec(comps):
        s = max(np.abs(ref[k]).max() for k in comps)
        return max(float(np.abs(mine[k] - ref[k]).max() / s) for k in comps)

    assert vec(("u", "v", "w")) < 1e-11
    assert vec(("ex", "ey", "ez")) < 1e-11
    for k in ("q", "phi"):
        assert np.abs(mine[k] - ref[k]).max() / np.abs(ref[k]).max() < 1e-11, k
    dev = np.abs(ref["rho"] - p.rho0).max()
    assert np.abs(mine["rho"] - ref["rho"]).max() / dev < 1e-10


def test_config0_inputs_regenerate():
    """The config-0 initial state (hydrostatic profile + seeded perturbation)
    is reproducible from the stored profile and the seed."""
    import make_golden as M
    g = golden("config0")
    p = M.case_params("config0")
    prof = {k: g[f"prof_{k}"] for k in O.FIELDS}
    f = O.state_from_profile(p, prof, seed=0, amp=1e-3)
    assert f["u"].shape == (33, 64, 64)
    assert np.all(f["u"][0] == 0) and np.all(f["w"][-1] == 0)
    assert 0.999e-3 < np.abs(f["w"][1:-1]).max() <= 1e-3
    # same seed -> same field, different seed -> different field
    f2 = O.state_from_profile(p, prof, seed=0, amp=1e-3)
    f3 = O.state_from_profile(p, prof, seed=1, amp=1e-3)
    assert np.array_equal(f["v"], f2["v"]) and not np.array_equal(f["v"], f3["v"])


def test_poisson_uniform_charge_free():
    """q = 0: phi is the linear profile and Ez = V/Lz everywhere (poisson.cu)."""
    p = O.params_from_groups(12, 10, 9, 1.5, 1.25, T=200, M=10, C=10, Fe=4000)
    o = O.Oracle(p)
    o.initialization()
    o.poisson()
    o.efield()
    f = o.get_fields()
    z = np.arange(p.nz)[:, None, None] * p.dz
    np.testing.assert_allclose(f["phi"], np.broadcast_to(p.voltage * (1 - z / p.lz), f["phi"].shape),
                               atol=1e-9 * p.voltage)
    np.testing.assert_allclose(f["ez"], p.voltage / p.lz, rtol=1e-11)
    assert np.abs(f["ex"]).max() < 1e-6 and np.abs(f["ey"]).max() < 1e-6


@pytest.mark.parametrize("m,n", [(1, 1), (2, 3), (5, 0)])
def test_poisson_manufactured_mode(m, n):
    """q = A sin(m pi z/(NZ-1)) cos(2 pi n x/Lx): phi = linear + A/(eps mu) * same mode with
    mu = kx^2 + (4/dz^2) sin^2(m pi/(2(NZ-1))), the discrete eigenvalue of
    poisson.cu:139."""
    p = O.params_from_groups(16, 8, 17, 2.0, 1.0, T=200, M=10, C=10, Fe=4000)
    o = O.Oracle(p)
    o.initialization()
    f = o.get_fields()
    z = np.arange(p.nz)[:, None, None]
    x = np.arange(p.nx)[None, None, :]
    A = 3.0
    kx = 2 * np.pi * n / p.lx
    mode = np.sin(m * np.pi * z / (p.nz - 1)) * np.cos(kx * x * p.dx) * np.ones((1, p.ny, 1))
    f["q"] = A * mode
    o.set_fields(f)
    o.poisson()
    phi = o.get_fields()["phi"]
    mu = kx ** 2 + 4 / p.dz ** 2 * np.sin(m * np.pi / (2 * (p.nz - 1))) ** 2
    expect = p.voltage * (1 - z * p.dz / p.lz) + A / (p.eps * mu) * mode
    np.testing.assert_allclose(phi, np.broadcast_to(expect, phi.shape), atol=1e-8 * p.voltage)


def thomas_poisson(p, q):
    """The product's formulation: 2D DFT in x, y, a tridiagonal solve in z per
    (kx, ky), inverse DFT.  Must equal the reference's odd-extension DFT solve."""
    nz = p.nz
    s = -q[1:nz - 1] / p.eps
    S = np.fft.fft2(s, axes=(1, 2))
    kx = np.fft.fftfreq(p.nx, d=1.0 / p.nx) * 2 * np.pi / p.lx
    ky = np.fft.fftfreq(p.ny, d=1.0 / p.ny) * 2 * np.pi / p.ly
    k2 = ky[:, None] ** 2 + kx[None, :] ** 2
    S[0, 0, 0] += -p.voltage / p.dz ** 2 * p.nx * p.ny  # Dirichlet lift on z = 1 (poisson.cu:97)
    n = nz - 2
    beta = 2 + k2 * p.dz ** 2
    d = S * p.dz ** 2
    cp = np.zeros((n,) + k2.shape)
    dp = np.zeros((n,) + k2.shape, complex)
    for i in range(n):
        prev_c = cp[i - 1] if i else 0.0
        prev_d = dp[i - 1] if i else 0.0
        cp[i] = 1.0 / (-beta - prev_c)
        dp[i] = (d[i] - prev_d) * cp[i]
    x = np.zeros_like(dp)
    x[n - 1] = dp[n - 1]
    for i in range(n - 2, -1, -1):
        x[i] = dp[i] - cp[i] * x[i + 1]
    phi = np.zeros(q.shape)
    phi[1:nz - 1] = np.fft.ifft2(x, axes=(1, 2)).real
    phi[0] = p.voltage
    return phi


@pytest.mark.parametrize("shape", [(16, 12, 9), (10, 15, 13), (8, 8, 33)])
def test_tridiagonal_solve_equals_odd_extension_dft(shape):
    nx, ny, nz = shape
    p = O.params_from_groups(nx, ny, nz, nx / (nz - 1), ny / (nz - 1), T=200, M=10, C=10, Fe=4000)
    rng = np.random.default_rng(7)
    o = O.Oracle(p)
    o.initialization()
    f = o.get_fields()
    f["q"] = 10.0 * rng.random((nz, ny, nx))
    o.set_fields(f)
    o.poisson()
    ref = o.get_fields()["phi"]
    mine = thomas_poisson(p, f["q"])
    assert relerr(mine, ref) < 1e-12


def random_state(p, seed):
    import make_golden as M
    return M.random_fields(p, seed)


def test_equilibrium_moments():
    """init_equilibrium (LBM.cu:110-276): sum f = rho, sum c f = rho u,
    sum g = q, sum c g = q (u + K E)."""
    p = O.reference_default_params(8, 6, 7)
    f = random_state(p, 3)
    o = O.Oracle(p)
    o.set_fields(f)
    f0, f1, h0, h1 = o.get_pops()
    F = np.concatenate([f0[None], f1])
    H = np.concatenate([h0[None], h1])
    np.testing.assert_allclose(F.sum(0), f["rho"], rtol=1e-14)
    np.testing.assert_allclose(H.sum(0), f["q"], rtol=1e-13)
    for a, (uk, ek) in enumerate((("u", "ex"), ("v", "ey"), ("w", "ez"))):
        mom = np.tensordot(EV[:, a], F, axes=1) / p.cfl
        np.testing.assert_allclose(mom, f["rho"] * f[uk], atol=1e-10 * p.rho0)
        momg = np.tensordot(EV[:, a], H, axes=1) / p.cfl
        np.testing.assert_allclose(momg, f["q"] * (f[uk] + p.K * f[ek]), atol=1e-11 * 10)


def test_collision_conserves_mass_and_charge():
    """TRT collide (LBM.cu:704-1089): per node, sum f and sum g unchanged; the
    Guo source adds F dt to the momentum."""
    p = O.params_from_groups(8, 6, 7, 1.0, 0.75, T=200, M=10, C=10, Fe=4000)
    f = random_state(p, 11)
    o = O.Oracle(p)
    o.set_fields(f)
    f0, f1, h0, h1 = o.get_pops()
    o.collide_only()
    g0, f2, k0, h2 = o.get_post()
    pre_f = f0 + f1.sum(0)
    pre_h = h0 + h1.sum(0)
    post_f = g0 + f2.sum(0)
    post_h = k0 + h2.sum(0)
    np.testing.assert_allclose(post_f[1:], pre_f[1:], rtol=1e-13)
    np.testing.assert_allclose(post_h[1:], pre_h[1:], rtol=1e-12, atol=1e-12)
    fld = o.get_fields()
    F = np.stack([fld["q"] * fld["ex"], fld["q"] * fld["ey"], fld["q"] * fld["ez"]])
    for a in range(3):
        pre = np.tensordot(EV[1:, a], f1, axes=1) / p.cfl
        post = np.tensordot(EV[1:, a], f2, axes=1) / p.cfl
        np.testing.assert_allclose((post - pre)[1:-1], (F[a] * p.dt)[1:-1],
                                   atol=1e-9 * np.abs(F[a] * p.dt).max() + 1e-9)


def test_wall_and_injection_rules():
    """gpu_boundary (LBM.cu:1103-1200) and gpu_bc_charge (LBM.cu:1320-1348)."""
    p = O.params_from_groups(6, 4, 7, 0.75, 0.5, T=200, M=10, C=10, Fe=4000, uw=0.02)
    o = O.Oracle(p)
    o.set_fields(random_state(p, 5))
    f0, f1, h0, h1 = o.get_pops()
    o.step_lbm()
    g0, f2, k0, h2 = o.get_post()
    _, f1n, k0n, h1n = o.get_pops()
    cs2 = 1 / 3 / p.cfl ** 2
    mw = {1: 1, 2: -1, 3: 1, 7: 1, 8: -1, 9: 1, 10: -1, 13: 1, 14: -1, 15: 1, 16: -1,
          19: 1, 20: -1, 21: 1, 22: -1, 23: 1, 24: -1, 25: -1, 26: 1}
    for d in range(1, 27):
        assert np.array_equal(f2[d - 1, 0], f1[opp(d) - 1, 0])  # bounce-back, lower plate
        m = 2 * p.rho0 * p.uw / cs2 * W[d] / p.cfl * mw.get(d, 0)
        np.testing.assert_allclose(f2[d - 1, -1], f1[opp(d) - 1, -1] + m, rtol=1e-15, atol=1e-13)
        assert np.array_equal(h2[d - 1, -1], h2[d - 1, -2])  # zero charge gradient
        np.testing.assert_allclose(h1n[d - 1, 0], -h2[opp(d) - 1, 0] + 2 * p.charge0 * W[d],
                                   rtol=1e-15, atol=1e-14)  # anti-bounce-back
    assert np.array_equal(g0[0], f0[0]) and np.array_equal(g0[-1], f0[-1])  # rest f restored
    # streaming: periodic pull in x, y, z of the post-wall populations
    for d in (5, 19, 26):
        e = EV[d]
        rolled = np.roll(f2[d - 1], shift=(e[2], e[1], e[0]), axis=(0, 1, 2))
        assert np.array_equal(f1n[d - 1], rolled)


def test_params_groups_roundtrip():
    p = O.params_from_groups(64, 64, 33, 2.0, 2.0, T=200, M=10, C=10, Fe=4000)
    assert abs(p.K - 2.5e-5) < 1e-18 and abs(p.nu - 0.125) < 1e-15
    assert abs(p.charge0 - 10.0) < 1e-12 and abs(p.diffu - 6.25e-5) < 1e-18
    g = O.groups_of(p)
    for k, v in dict(T=200, M=10, C=10, Fe=4000).items():
        assert abs(g[k] - v) < 1e-9 * v
    ref = O.groups_of(O.reference_default_params())
    assert abs(ref["T"] - 996.0) < 1.0 and abs(ref["M"] - 10) < 1e-9  # LBM.cu:1375-1378


def test_column_state_broadcast_evolves_as_the_column_and_its_fields_do_not():
    """The restatement behind ehd_set_state_from_column, in the reference's own
    scheme: a 1 x 1 x NZ column's populations broadcast over x, y evolve as the
    column does; equilibrium populations rebuilt from its fields do not (the
    injector alternates with period two, and its planes carry non-equilibrium
    parts the rebuild drops)."""
    p = O.params_from_groups(4, 4, 9, 0.5, 0.5, T=300, M=10, C=10, Fe=4000,
                             lambda_f=1.0 / 12.0, lambda_g=1e-6)
    q = O.Params(**{k: getattr(p, k) for k, _ in O.Params._fields_})
    q.nx, q.ny, q.lx, q.ly = 1, 1, p.dx, p.dy
    col = O.Oracle(q)
    col.initialization()
    col.step(2000)
    f = col.get_fields()
    f0, f1, h0, h1 = col.get_pops()
    shape = (p.nz, p.ny, p.nx)
    bc = {k: np.broadcast_to(v, shape) for k, v in f.items()}
    a = O.Oracle(p)
    a.set_fields(bc)
    a.set_pops(np.broadcast_to(f0, shape), np.broadcast_to(f1, (26,) + shape),
               np.broadcast_to(h0, shape), np.broadcast_to(h1, (26,) + shape))
    b = O.Oracle(p)
    b.set_fields(bc)
    for o in (a, b, col):
        o.step(50)
    ref = {k: np.broadcast_to(v, shape) for k, v in col.get_fields().items()}
    ga, gb = a.get_fields(), b.get_fields()
    for k in ("rho", "q", "phi"):
        assert relerr(ga[k], ref[k]) < 1e-12, k
    assert relerr(gb["q"], ref["q"]) > 1e-3
