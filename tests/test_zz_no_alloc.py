"""ehd_poisson_noalloc: the Poisson solve for callers that cannot allocate.

Some callers cannot call cudaMalloc (their GPU memory belongs to another
framework's pool, or an allocation would synchronise a pipeline they run
inside).  ehd_poisson_noalloc gives them the Poisson solve and E field on
device arrays they own, with its working storage in a fixed file-scope device
array.  This test calls it through the C ABI twice in a row, on two different
charge fields, and checks each result against the context entry points
(ehd_set_fields + ehd_poisson + ehd_get_fields) with the FP64 tolerance of the
other Poisson tests.  The second call checks that nothing left in the shared
array by the first call leaks into the next result, and that it allocates
nothing: the device's free memory and torch's reserved memory are the same
before and after it.  Collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

from conftest import O, ehd, relerr

pytestmark = pytest.mark.gpu


def to_ehd(p):
    return ehd.Params.from_dict(p.as_dict())


def vec_err(a, b, comps):
    scale = max(np.abs(b[k]).max() for k in comps)
    return max(float(np.abs(a[k] - b[k]).max() / scale) for k in comps)


def test_poisson_noalloc_matches_context_path_twice():
    import torch
    import make_golden as M

    dz = 1.0 / 32
    # nx = 64 takes the compile-time-radix FFT, ny = 48 the run-time radix one
    p = O.params_from_groups(64, 48, 33, 64 * dz, 48 * dz, T=200, M=10, C=10, Fe=4000)
    pe = to_ehd(p)
    for seed in (11, 12):
        f = M.random_fields(p, seed)
        with ehd.Simulation(pe, "fp64") as sim:
            sim.set_fields(f)
            sim.poisson()
            ref = sim.get_fields()
        q = torch.from_numpy(np.ascontiguousarray(f["q"])).cuda()
        out = {k: torch.full_like(q, float("nan")) for k in ("phi", "ex", "ey", "ez")}
        torch.cuda.synchronize()
        before = (torch.cuda.mem_get_info()[0], torch.cuda.memory_reserved())
        rc = ehd.lib().ehd_poisson_noalloc(ctypes.byref(pe), q.data_ptr(),
                                           out["phi"].data_ptr(), out["ex"].data_ptr(),
                                           out["ey"].data_ptr(), out["ez"].data_ptr(), None)
        torch.cuda.synchronize()
        assert rc == 0, ehd.lib().ehd_last_error()
        if seed == 12:  # the array is committed by the first call; later calls allocate nothing
            assert (torch.cuda.mem_get_info()[0], torch.cuda.memory_reserved()) == before
        mine = {k: v.cpu().numpy() for k, v in out.items()}
        assert relerr(mine["phi"], ref["phi"]) < 1e-11
        assert vec_err(mine, ref, ("ex", "ey", "ez")) < 1e-11


def test_poisson_noalloc_rejects_grids_beyond_its_storage():
    import torch

    p = O.params_from_groups(512, 512, 129, 4.0, 4.0, T=200, M=10, C=10, Fe=4000)
    pe = to_ehd(p)
    d = torch.zeros(8, dtype=torch.float64, device="cuda")  # never touched
    rc = ehd.lib().ehd_poisson_noalloc(ctypes.byref(pe), d.data_ptr(), d.data_ptr(),
                                       d.data_ptr(), d.data_ptr(), d.data_ptr(), None)
    assert rc == -1
    assert b"EHD_NOALLOC_SCRATCH_BYTES" in ehd.lib().ehd_last_error()
