"""The C++ driver (ehd_sim, the host program the reference's main.cu is)."""
import subprocess

import numpy as np
import pytest

from conftest import O, PKG, ehd

pytestmark = pytest.mark.gpu


def test_driver_matches_the_api(tmp_path):
    exe = PKG / "ehd_sim"
    assert exe.exists(), "build with make -C ehd-convection-3d_b200"
    r = subprocess.run([str(exe), "--nx", "16", "--ny", "16", "--nz", "9", "--steps", "20",
                        "--current-every", "5", "--save-every", "10", "--dmd-every", "10",
                        "--precision", "fp64"],
                       cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert "speed:" in r.stdout and r.stdout.count("Current = ") == 4
    # uz files for DMD at i % 10 == 1, named by the time after that step
    assert r.stdout.count("Iteration: ") == 2
    dmd = sorted(f.name for f in tmp_path.glob("*.dat")
                 if f.name not in ("data.dat", "data_end.dat", "umax.dat"))
    assert len(dmd) == 2, dmd
    for f in dmd:
        assert np.loadtxt(tmp_path / f).shape == (16 * 16 * 9, 2)
    # the same run through the API: the reference defaults, its initialization
    p = O.reference_default_params(16, 16, 9)
    with ehd.Simulation(ehd.Params.from_dict(p.as_dict()), "fp64") as sim:
        sim.initialize()
        sim.step(20)
        sim.write_data_end(tmp_path / "api_end.dat")
    a = np.loadtxt(tmp_path / "data_end.dat")
    b = np.loadtxt(tmp_path / "api_end.dat")
    assert a.shape == b.shape == (16 * 16 * 9, 10)
    assert np.array_equal(a, b)
    text = (tmp_path / "data.dat").read_text()
    assert text.count("ZONE T=") == 4  # initial, i % 10 == 1 twice, final
    assert len((tmp_path / "umax.dat").read_text().splitlines()) == 5
