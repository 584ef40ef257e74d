"""Fine-grid warm start (finestart.py), host side: the periodic tiling and
linear interpolation that carry a coarse prediction to the fine grid, and the
fine grid's parameters."""
import importlib.util

import numpy as np
import pytest

from conftest import PKG, ehd


def _finestart():
    spec = importlib.util.spec_from_file_location("ehd_finestart", PKG / "finestart.py")
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


F = _finestart()


def test_upsample_shape_keeps_coarse_nodes_and_tiles_periodically():
    rng = np.random.default_rng(0)
    c = rng.standard_normal((9, 12, 16))
    f = F.upsample(c, tiles=2, factor=4)
    assert f.shape == (33, 96, 128)
    # every coarse node, in both tiles along x and y
    for ty in range(2):
        for tx in range(2):
            blk = f[::4, ty * 48:(ty + 1) * 48:4, tx * 64:(tx + 1) * 64:4]
            assert np.array_equal(blk, c)


def test_upsample_is_exact_for_fields_linear_between_nodes():
    nz, ny, nx = 5, 6, 8
    z = np.arange(nz)[:, None, None] * 1.0
    c = np.broadcast_to(2.0 + 0.5 * z, (nz, ny, nx))
    f = F.upsample(c, tiles=1, factor=3)
    zf = np.arange(f.shape[0])[:, None, None] / 3.0
    assert np.allclose(f, 2.0 + 0.5 * zf, rtol=0, atol=1e-14)
    # periodic x: the point halfway between the last node and the first
    c = np.zeros((2, 1, nx))
    c[:, :, -1] = 1.0
    f = F.upsample(c, tiles=1, factor=2)
    assert f[0, 0, -1] == pytest.approx(0.5) and f[0, 0, -2] == pytest.approx(1.0)
    assert f[0, 0, -3] == pytest.approx(0.5) and f[0, 0, 0] == pytest.approx(0.0)


def test_upsample_of_a_box_periodic_wave_is_the_same_wave_on_the_wider_box():
    nx = 16
    x = np.arange(nx) / nx
    c = np.broadcast_to(np.sin(2 * np.pi * x), (3, 1, nx))
    f = F.upsample(c, tiles=2, factor=1)
    xf = np.arange(2 * nx) / nx
    assert np.allclose(f[0, 0], np.sin(2 * np.pi * xf), atol=1e-12)


def test_fine_params_refine_the_grid_and_keep_the_physics():
    p = ehd.params_from_groups(16, 16, 9, 2.0, 2.0, T=300, M=10, C=10, Fe=4000,
                               lambda_f=1.0 / 12.0, lambda_g=1e-6)
    q = F.fine_params(ehd, p, tiles=2, factor=4)
    assert (q.nx, q.ny, q.nz) == (128, 128, 33)
    assert q.lx == pytest.approx(4.0) and q.lz == pytest.approx(1.0)
    assert q.dz == pytest.approx(1.0 / 32) and q.dx == pytest.approx(q.lx / q.nx)
    assert q.dt == pytest.approx(q.cfl * q.dz)
    for k in ("nu", "K", "diffu", "charge0", "voltage", "eps", "rho0", "lambda_f", "lambda_g"):
        assert getattr(q, k) == getattr(p, k), k
    gp, gq = ehd.groups_of(p), ehd.groups_of(q)
    for k in ("T", "M", "C", "Fe"):
        assert gq[k] == pytest.approx(gp[k], rel=1e-12), k


def test_warm_fields_hold_the_walls_and_the_fine_hydrostatic_density():
    rng = np.random.default_rng(1)
    pred = {k: rng.standard_normal((5, 4, 4)) for k in F.PRED_FIELDS}
    prof = {"rho": np.linspace(1600.0, 1601.0, 9)}
    f = F.warm_fields(pred, prof, tiles=1, factor=2)
    assert f["q"].shape == (9, 8, 8)
    for k in ("u", "v", "w"):
        assert not f[k][0].any() and not f[k][-1].any()
    assert np.array_equal(f["rho"][:, 3, 5], prof["rho"])
    assert not f["ex"].any() and f["phi"][::2, ::2, ::2] == pytest.approx(pred["phi"])
