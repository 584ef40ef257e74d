"""The bulk-copy row kernel (steady-state steps with FP32 or FP64 populations
on grids with 32 <= nx <= 256 and rows of a multiple of 16 bytes; CTAs of nx
rounded up to whole warps, the lanes past the row idle) against the oracle and
against the one-thread-per-node kernel.

The first step after set_fields always runs on the per-node kernel (it reads
the uploaded state in place); the steps after it run on the row kernel
wherever it applies, so these cases chain the two and check the chain.
"""
import numpy as np
import pytest

from conftest import O, ehd, relerr

pytestmark = pytest.mark.gpu


def to_ehd(p):
    return ehd.Params.from_dict(p.as_dict())


def random_fields(p, seed):
    import make_golden as M
    return M.random_fields(p, seed)


# x-rows of 1 to 8 warps, and rows that end inside a warp (48, 80, 100, 250
# nodes); ny = 1 and nz = 4 are the smallest planes and stacks
@pytest.mark.parametrize("shape", [(32, 12, 9), (64, 20, 11), (96, 10, 6), (256, 4, 5),
                                   (128, 1, 17), (64, 64, 4), (48, 12, 9), (80, 10, 7),
                                   (100, 6, 5), (250, 3, 5)])
def test_row_kernel_steps_match_oracle(shape):
    nx, ny, nz = shape
    dz = 1.0 / (nz - 1)
    p = O.params_from_groups(nx, ny, nz, nx * dz, ny * dz, T=200, M=10, C=10, Fe=4000,
                             exf=50.0, uw=0.01)
    f = random_fields(p, 23)
    o = O.Oracle(p)
    o.set_fields(f)
    with ehd.Simulation(to_ehd(p), "fp64") as sim:
        sim.set_fields(f)
        sim.step(1)
        sim.step(6)  # six steps on the row kernel
        o.step(7)
        a, b = sim.get_fields(), o.get_fields()
    for k in O.FIELDS:
        assert relerr(a[k], b[k]) < 1e-10, (k, relerr(a[k], b[k]))


@pytest.mark.parametrize("shape", [(64, 64, 33), (80, 48, 25)])
@pytest.mark.parametrize("prec,tol", [("fp64", 1e-11), ("fp32", 1e-5)])
def test_row_kernel_agrees_with_node_kernel(shape, prec, tol):
    """Same run on both kernels (80 nodes: the third warp of a row half
    idle).  The plane sums behind the per-plane references are taken in a
    different order, so the two agree to the rounding of the storage type,
    not bitwise."""
    nx, ny, nz = shape
    dz = 1.0 / (nz - 1)
    p = O.params_from_groups(nx, ny, nz, nx * dz, ny * dz, T=200, M=10, C=10, Fe=4000)
    f = random_fields(p, 5)
    out = []
    for rows in (True, False):
        with ehd.Simulation(to_ehd(p), prec, row_kernel=rows) as sim:
            sim.set_fields(f)
            sim.step(40)
            out.append((sim.get_fields(), sim.diagnostics()))
    for k in ("rho", "q", "phi"):
        assert relerr(out[0][0][k], out[1][0][k]) < tol, (k, relerr(out[0][0][k], out[1][0][k]))
    scale = max(np.abs(out[1][0][k]).max() for k in ("u", "v", "w"))
    for k in ("u", "v", "w"):
        assert np.abs(out[0][0][k] - out[1][0][k]).max() / scale < tol, k
    assert out[0][1]["current"] == pytest.approx(out[1][1]["current"], rel=tol)


def test_row_kernel_graphs_and_direct_launches_agree_bitwise():
    dz = 1.0 / 16
    p = O.params_from_groups(128, 32, 17, 128 * dz, 32 * dz, T=200, M=10, C=10, Fe=4000)
    f = random_fields(p, 9)
    out = []
    for graphs in (True, False):
        with ehd.Simulation(to_ehd(p), "fp32", graphs=graphs) as sim:
            sim.set_fields(f)
            sim.step(9)
            sim.step(4)
            out.append(sim.get_fields())
    for k in O.FIELDS:
        assert np.array_equal(out[0][k], out[1][k]), k


def test_contexts_of_different_sizes_share_kernels():
    """Kernel attributes are per function, not per context: contexts of
    different widths created one after the other (the larger first) must all
    still launch.  96- and 64-wide FP32 grids share the row kernel; 480- and
    384-wide FP64 grids share the run-time-radix row FFT, each with more than
    48 KB of shared memory."""
    cases = [((96, 16, 9), "fp32"), ((64, 16, 9), "fp32"), ((480, 6, 5), "fp64"),
             ((384, 6, 5), "fp64")]
    sims, refs = [], []
    for (nx, ny, nz), prec in cases:
        dz = 1.0 / (nz - 1)
        p = O.params_from_groups(nx, ny, nz, nx * dz, ny * dz, T=200, M=10, C=10, Fe=4000)
        f = random_fields(p, 7)
        sim = ehd.Simulation(to_ehd(p), prec)
        sim.set_fields(f)
        sims.append(sim)
        o = O.Oracle(p)
        o.set_fields(f)
        o.step(3)
        refs.append(o.get_fields())
    try:
        for k in range(3):
            for sim in sims:
                sim.step(1)
        for ((shape, prec), sim, ref) in zip(cases, sims, refs):
            out = sim.get_fields()
            tol = 1e-10 if prec == "fp64" else 1e-5
            for k in ("q", "phi"):
                assert relerr(out[k], ref[k]) < tol, (shape, prec, k, relerr(out[k], ref[k]))
    finally:
        for sim in sims:
            sim.close()
