"""Fine-grid warm start (finestart.py) end to end on small grids: a network's
coarse prediction, saved and reloaded, tiled and interpolated onto a grid
twice as fine and twice as wide, run with FP16 deviation storage beside the
same start in FP32 and a cold FP32 start."""
import importlib.util
import math

import numpy as np
import pytest

from conftest import PKG, ehd, fno

pytestmark = pytest.mark.gpu


def _finestart():
    spec = importlib.util.spec_from_file_location("ehd_finestart", PKG / "finestart.py")
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def test_fine_grid_warm_start_runs_and_stays_close_to_fp32(tmp_path):
    F = _finestart()
    import torch
    net = fno.FNO(16, 16, 9, 9, 5, width=8, layers=2, modes=(4, 4, 4), hidden=16, max_batch=1,
                  seed=3)
    # outputs near zero velocity and near zero change of q and phi: the start's
    # column carried over, a smooth, finite start
    mean = np.array([0.0, 0.0, 0.0, 0.0, 0.0])
    std = np.array([1e-4, 1e-4, 1e-4, 1e-3, 1e-3])
    path = tmp_path / "net.npz"
    F.save_net(path, net, mean, std)
    net2, m2, s2 = F.load_net(path)
    assert np.array_equal(net2.params(), net.params())
    assert np.array_equal(m2, mean) and np.array_equal(s2, std)
    x = torch.randn(1, 9, 16, 16, 9, device="cuda")
    assert torch.equal(net.forward(x), net2.forward(x))
    net.close()

    group = {"T": 300.0, "M": 10.0, "C": 10.0, "seed": 5}
    cp, pred = F.predict(ehd, net2, m2, s2, group, (16, 16, 9))
    net2.close()
    assert pred["q"].shape == (9, 16, 16)
    q = pred["q"]
    assert np.all(np.isfinite(q)) and q.min() > -1e-2 * cp.charge0
    # each plane is the column's value plus a change of order std
    assert np.all(np.abs(q - q.mean(axis=(1, 2), keepdims=True)) < 1e-2 * cp.charge0)
    assert np.ptp(q.mean(axis=(1, 2))) > 0.1 * cp.charge0
    res = F.compare(ehd, cp, pred, group, tiles=2, factor=2, steps=40, sample=20,
                    warm_precision="fp16")
    assert res["fine_grid"] == [64, 64, 17] and res["fine_lx"] == pytest.approx(2 * cp.lx)
    for name in ("warm_fp16", "warm_fp32", "cold_fp32"):
        h = res[name]["history"]
        assert [r["step"] for r in h] == [20, 40], name
        assert not any(r["nonfinite"] for r in h), name
        assert all(math.isfinite(r["kinetic_energy"]) and math.isfinite(r["nu_e"]) for r in h)
        assert res[name]["mlups"] > 0
    # both warm runs start from the same fields
    assert res["warm_fp16"]["initial"]["total_charge"] == pytest.approx(
        res["warm_fp32"]["initial"]["total_charge"], rel=1e-3)
    # the warm start carries the interpolated charge, the cold start the
    # hydrostatic one: their total charges differ
    assert res["warm_fp32"]["initial"]["total_charge"] != pytest.approx(
        res["cold_fp32"]["initial"]["total_charge"], rel=1e-3)
    err = res["warm_storage_error"]
    assert set(err) == {"u", "v", "w", "q", "phi"}
    assert err["q"] < 1e-2 and err["phi"] < 1e-2, err
