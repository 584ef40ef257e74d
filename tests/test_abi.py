"""The C-ABI library: builds, loads, exports every declared symbol, and
validates arguments on the host.  CPU only -- no call here touches a GPU."""
import ctypes
import re
import subprocess

import pytest

from conftest import O, ROOT, ehd, has_gpu

HEADER = ROOT / "include" / "ehd.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ehd_[a-z_0-9]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    names = declared_functions()
    assert len(names) >= 15
    out = subprocess.run(["nm", "-D", "--defined-only", str(ehd.LIB_PATH)], capture_output=True,
                         text=True, check=True).stdout
    exported = set(re.findall(r"\bT (ehd_\w+)", out))
    missing = [n for n in names if n not in exported]
    assert not missing, missing
    L = ehd.lib()
    for n in names:
        assert getattr(L, n) is not None


def test_binding_covers_the_header():
    assert sorted(ehd.SIGNATURES) == declared_functions()


def test_abi_version():
    assert ehd.lib().ehd_abi_version() == 1


def test_params_from_groups_matches_reference_formula():
    p = ehd.params_from_groups(64, 64, 33, 2.0, 2.0, T=200, M=10, C=10, Fe=4000)
    q = O.params_from_groups(64, 64, 33, 2.0, 2.0, T=200, M=10, C=10, Fe=4000)
    for k in ("K", "nu", "charge0", "diffu", "dt", "dx", "dz"):
        assert getattr(p, k) == pytest.approx(getattr(q, k), rel=1e-15), k
    g = ehd.groups_of(p)
    assert g["T"] == pytest.approx(200) and g["Fe"] == pytest.approx(4000)


@pytest.mark.parametrize("bad", [dict(nz=3), dict(nx=-4), dict(ny=0), dict(dt=0.0), dict(nu=-1.0),
                                 dict(lambda_g=0.0), dict(pad_=1), dict(nx=1 << 16, ny=1 << 16)])
def test_create_rejects_bad_params(bad):
    p = ehd.params_from_groups(16, 16, 9, 2.0, 2.0, T=200, M=10, C=10, Fe=4000)
    for k, v in bad.items():
        setattr(p, k, v)
    h = ctypes.c_void_p()
    cfg = ehd.Config(precision=1)
    rc = ehd.lib().ehd_create(ctypes.byref(p), ctypes.byref(cfg), ctypes.byref(h))
    assert rc == -1 and not h.value
    assert ehd.lib().ehd_last_error()


def test_create_rejects_bad_precision():
    p = ehd.params_from_groups(16, 16, 9, 2.0, 2.0, T=200, M=10, C=10, Fe=4000)
    h = ctypes.c_void_p()
    cfg = ehd.Config(precision=9)
    assert ehd.lib().ehd_create(ctypes.byref(p), ctypes.byref(cfg), ctypes.byref(h)) == -1


def test_null_arguments_are_errors_not_crashes():
    L = ehd.lib()
    assert L.ehd_step(None, 1) == -1
    assert L.ehd_destroy(None) == 0
    assert L.ehd_synchronize(None) == -1
    assert L.ehd_diagnostics(None, None) == -1
    assert L.ehd_create(None, None, None) == -1
    assert L.ehd_hydrostatic_column(None, None, 10, None, None) == -1
    assert L.ehd_set_state_from_column(None, None, 0, 0.0) == -1
    assert L.ehd_write_dmd(None, b"x.dat") == -1
    # checked before any CUDA call
    assert L.ehd_poisson_noalloc(None, None, None, None, None, None, None) == -1


@pytest.mark.skipif(has_gpu(), reason="checks the no-GPU error path")
def test_create_without_gpu_reports_cuda_error():
    p = ehd.params_from_groups(16, 16, 9, 2.0, 2.0, T=200, M=10, C=10, Fe=4000)
    with pytest.raises(ehd.EhdError) as e:
        ehd.Simulation(p, "fp32")
    assert e.value.code in (-1, -2)


def test_fno_header_is_exported_and_bound():
    from conftest import fno
    text = re.sub(r"/\*.*?\*/", "", (ROOT / "include" / "ehd_fno.h").read_text(), flags=re.S)
    names = sorted(set(re.findall(r"\b(ehd_[a-z_0-9]+)\s*\(", text)))
    assert len(names) >= 10
    out = subprocess.run(["nm", "-D", "--defined-only", str(ehd.LIB_PATH)], capture_output=True,
                         text=True, check=True).stdout
    exported = set(re.findall(r"\bT (ehd_\w+)", out))
    assert not [n for n in names if n not in exported]
    assert sorted(fno.SIGNATURES) == names
    fno.lib()  # binds every signature
