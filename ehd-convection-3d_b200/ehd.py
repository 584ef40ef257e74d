"""Python binding of libehd.so (include/ehd.h) through ctypes.

This is the host-side mirror used by the tests and the benchmark: one
``Simulation`` is one ``ehd_ctx``.  Field arrays are numpy float64 of shape
(nz, ny, nx), the reference layout x + NX*(y + NY*z) (LBM.cu:21-24).  The
binding adds no computation of its own: every call goes to the CUDA library,
and a missing library is an error (there is no CPU path).
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libehd.so"

FIELDS = ("rho", "u", "v", "w", "q", "phi", "ex", "ey", "ez")
PRECISIONS = {"fp64": 0, "fp32": 1, "fp16": 2, "bf16": 3, "mixed": 4}
FLAG_NO_GRAPH = 0x1
FLAG_NODE_KERNEL = 0x2


class EhdError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"ehd error {code}: {msg}")
        self.code = code


class Params(ctypes.Structure):
    """ehd_params (include/ehd.h)."""

    _fields_ = [
        ("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("nz", ctypes.c_int32),
        ("pad_", ctypes.c_int32),
        ("lx", ctypes.c_double), ("ly", ctypes.c_double), ("lz", ctypes.c_double),
        ("dx", ctypes.c_double), ("dy", ctypes.c_double), ("dz", ctypes.c_double),
        ("dt", ctypes.c_double), ("cfl", ctypes.c_double),
        ("rho0", ctypes.c_double), ("charge0", ctypes.c_double),
        ("voltage", ctypes.c_double), ("eps", ctypes.c_double),
        ("diffu", ctypes.c_double), ("nu", ctypes.c_double), ("K", ctypes.c_double),
        ("uw", ctypes.c_double), ("exf", ctypes.c_double),
        ("lambda_f", ctypes.c_double), ("lambda_g", ctypes.c_double),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "pad_"}

    @classmethod
    def from_dict(cls, d):
        p = cls()
        for k, v in d.items():
            setattr(p, k, v)
        p.pad_ = 0
        return p


class Config(ctypes.Structure):
    _fields_ = [("precision", ctypes.c_int32), ("device", ctypes.c_int32),
                ("stream", ctypes.c_void_p), ("flags", ctypes.c_uint32),
                ("reserved", ctypes.c_uint32 * 7)]


class Diag(ctypes.Structure):
    _fields_ = [("current", ctypes.c_double), ("nu_e", ctypes.c_double),
                ("kinetic_energy", ctypes.c_double), ("total_charge", ctypes.c_double),
                ("umax", ctypes.c_double), ("time", ctypes.c_double),
                ("step", ctypes.c_int64), ("nonfinite", ctypes.c_int32),
                ("pad_", ctypes.c_int32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "pad_"}


class Tuning(ctypes.Structure):
    _fields_ = [("lbm_kernel", ctypes.c_int32), ("node_block_x", ctypes.c_int32),
                ("fft_rows", ctypes.c_int32), ("fft_cols", ctypes.c_int32),
                ("poisson_path", ctypes.c_int32), ("z_solve", ctypes.c_int32),
                ("reserved", ctypes.c_int32 * 2)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}


# every symbol include/ehd.h declares, with (restype, argtypes)
_dp = ctypes.POINTER(ctypes.c_double)
_vp = ctypes.c_void_p
_i = ctypes.c_int
SIGNATURES = {
    "ehd_abi_version": (_i, []),
    "ehd_last_error": (ctypes.c_char_p, []),
    "ehd_create": (_i, [ctypes.POINTER(Params), ctypes.POINTER(Config), ctypes.POINTER(_vp)]),
    "ehd_destroy": (_i, [_vp]),
    "ehd_set_fields": (_i, [_vp] + [_dp] * 9),
    "ehd_initialize": (_i, [_vp]),
    "ehd_get_fields": (_i, [_vp] + [_dp] * 9),
    "ehd_step": (_i, [_vp, _i]),
    "ehd_stream_collide_save": (_i, [_vp]),
    "ehd_poisson": (_i, [_vp]),
    "ehd_synchronize": (_i, [_vp]),
    "ehd_current": (_i, [_vp, _dp]),
    "ehd_set_reference_current": (_i, [_vp, ctypes.c_double]),
    "ehd_diagnostics": (_i, [_vp, ctypes.POINTER(Diag)]),
    "ehd_device_bytes": (_i, [_vp, ctypes.POINTER(ctypes.c_size_t)]),
    "ehd_params_from_groups": (_i, [ctypes.POINTER(Params)] + [ctypes.c_double] * 4),
    "ehd_groups_from_params": (_i, [ctypes.POINTER(Params)] + [_dp] * 4),
    "ehd_poisson_noalloc": (_i, [ctypes.POINTER(Params), _vp, _vp, _vp, _vp, _vp, _vp]),
    "ehd_hydrostatic_profile": (_i, [ctypes.POINTER(Params), ctypes.POINTER(Config), _i, _dp, _dp]),
    "ehd_set_state_seeded": (_i, [_vp, _dp, ctypes.c_uint64, ctypes.c_double]),
    "ehd_run_to_saturation": (_i, [_vp, _i, ctypes.c_double, _i, ctypes.c_int64, _dp,
                                   ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(_i)]),
    "ehd_checkpoint": (_i, [_vp, ctypes.c_char_p]),
    "ehd_restore": (_i, [_vp, ctypes.c_char_p]),
    "ehd_write_data_end": (_i, [_vp, ctypes.c_char_p]),
    "ehd_read_data_end": (_i, [_vp, ctypes.c_char_p]),
    "ehd_write_tecplot": (_i, [_vp, ctypes.c_char_p, _i]),
    "ehd_get_tuning": (_i, [_vp, ctypes.POINTER(Tuning)]),
    "ehd_set_tuning": (_i, [_vp, ctypes.POINTER(Tuning)]),
    "ehd_batch_create": (_i, [ctypes.POINTER(Params), _i, ctypes.POINTER(Config),
                              ctypes.POINTER(_vp)]),
    "ehd_batch_destroy": (_i, [_vp]),
    "ehd_batch_size": (_i, [_vp]),
    "ehd_batch_instance": (_i, [_vp, _i, ctypes.POINTER(_vp)]),
    "ehd_batch_set_active": (_i, [_vp, _i, _i]),
    "ehd_batch_set_mode": (_i, [_vp, _i]),
    "ehd_batch_step": (_i, [_vp, _i]),
    "ehd_batch_run_to_saturation": (_i, [_vp, _i, ctypes.c_double, _i, ctypes.c_int64,
                                         ctypes.POINTER(ctypes.c_int32),
                                         ctypes.POINTER(ctypes.c_int64), _dp]),
    "ehd_batch_autotune": (_i, [_vp, _i]),
    "ehd_hydrostatic_column": (_i, [ctypes.POINTER(Params), ctypes.POINTER(Config), _i,
                                    ctypes.POINTER(_vp), ctypes.POINTER(ctypes.c_double)]),
    "ehd_set_state_from_column": (_i, [_vp, _vp, ctypes.c_uint64, ctypes.c_double]),
    "ehd_write_dmd": (_i, [_vp, ctypes.c_char_p]),
}

_lib = None


def lib():
    """Load libehd.so; raise if it was not built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise FileNotFoundError(
                f"{LIB_PATH} is missing: build it with `make -C {HERE}` (no CPU fallback)")
        L = ctypes.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _check(rc):
    if rc != 0:
        raise EhdError(rc, lib().ehd_last_error().decode(errors="replace"))


def _ptr(a):
    return a.ctypes.data_as(_dp)


def params_from_groups(nx, ny, nz, lx, ly, T, M, C, Fe, lambda_f=0.25, lambda_g=0.25,
                       cfl=0.01, lz=1.0, **over) -> Params:
    """Grid + dimensionless groups -> ehd_params, through ehd_params_from_groups
    (the inverse of the reference's compute_parameters, LBM.cu:1356-1379)."""
    dz = lz / (nz - 1)
    p = Params(nx=nx, ny=ny, nz=nz, pad_=0, lx=lx, ly=ly, lz=lz, dx=lx / nx, dy=ly / ny, dz=dz,
               dt=cfl * dz, cfl=cfl, rho0=1600.0, charge0=0.0, voltage=1.0e4, eps=1.0e-4,
               diffu=0.0, nu=0.0, K=0.0, uw=0.0, exf=0.0, lambda_f=lambda_f, lambda_g=lambda_g)
    _check(lib().ehd_params_from_groups(ctypes.byref(p), T, M, C, Fe))
    for k, v in over.items():
        setattr(p, k, v)
    return p


def poisson_noalloc(p: Params, q, phi, ex, ey, ez, stream=None):
    """ehd_poisson_noalloc on device buffers given as integer device addresses
    (e.g. torch ``tensor.data_ptr()``): q in; phi, ex, ey, ez out.  For callers
    that cannot allocate device memory; asynchronous on `stream`."""
    _check(lib().ehd_poisson_noalloc(ctypes.byref(p), q, phi, ex, ey, ez, stream))


def hydrostatic_profile(p: Params, nsteps: int, precision: str = "fp64", device: int = 0):
    """The u = 0 steady state of the step on a 1 x 1 x NZ column after nsteps
    steps: (profile dict of per-z arrays, I0 on the full NX x NY plane)."""
    prof = np.empty(9 * p.nz, np.float64)
    i0 = ctypes.c_double()
    cfg = Config(precision=PRECISIONS[precision], device=device)
    _check(lib().ehd_hydrostatic_profile(ctypes.byref(p), ctypes.byref(cfg), int(nsteps),
                                         _ptr(prof), ctypes.byref(i0)))
    return {k: prof[i * p.nz:(i + 1) * p.nz].copy() for i, k in enumerate(FIELDS)}, i0.value


def hydrostatic_column(p: Params, nsteps: int, precision: str = "fp64", device: int = 0):
    """ehd_hydrostatic_column: (the 1 x 1 x NZ column after nsteps + 1 steps
    as a Simulation, I0 on the full NX x NY plane).  Close the column when
    done with it."""
    q = Params.from_dict(p.as_dict())
    q.nx, q.ny, q.lx, q.ly = 1, 1, p.dx, p.dy
    h = _vp()
    i0 = ctypes.c_double()
    cfg = Config(precision=PRECISIONS[precision], device=device)
    _check(lib().ehd_hydrostatic_column(ctypes.byref(p), ctypes.byref(cfg), int(nsteps),
                                        ctypes.byref(h), ctypes.byref(i0)))
    col = Simulation._view(h, q)
    col.owned = True
    return col, i0.value


def groups_of(p: Params):
    out = [ctypes.c_double() for _ in range(4)]
    _check(lib().ehd_groups_from_params(ctypes.byref(p), *[ctypes.byref(o) for o in out]))
    return dict(zip(("T", "M", "C", "Fe"), [o.value for o in out]))


def _sampled(sims, n: int, step) -> list:
    if n < 1:
        raise ValueError("n must be >= 1")
    first = None
    if n >= 2:
        step(n - 1)
        first = [s.diagnostics()["current"] for s in sims]
    step(1)
    out = []
    for k, s in enumerate(sims):
        d = s.diagnostics()
        mean = d["current"] if first is None else 0.5 * (first[k] + d["current"])
        if d["current"] != 0.0:  # nu_e = current / I0
            d["nu_e"] *= mean / d["current"]
        d["current_mean"] = mean
        out.append(d)
    return out


class Simulation:
    """One simulation instance (ehd_ctx) on one GPU."""

    def __init__(self, params: Params, precision: str = "fp32", device: int = 0,
                 stream: int | None = None, graphs: bool = True, row_kernel: bool = True):
        self.p = params
        self.shape = (params.nz, params.ny, params.nx)
        flags = (0 if graphs else FLAG_NO_GRAPH) | (0 if row_kernel else FLAG_NODE_KERNEL)
        cfg = Config(precision=PRECISIONS[precision], device=device, stream=stream,
                     flags=flags)
        h = _vp()
        _check(lib().ehd_create(ctypes.byref(params), ctypes.byref(cfg), ctypes.byref(h)))
        self.h = h
        self.owned = True

    @classmethod
    def _view(cls, handle, params: Params):
        """A context owned by someone else (a Batch instance)."""
        sim = cls.__new__(cls)
        sim.p = params
        sim.shape = (params.nz, params.ny, params.nx)
        sim.h = handle
        sim.owned = False
        return sim

    def close(self):
        if getattr(self, "h", None):
            if getattr(self, "owned", True):
                lib().ehd_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_fields(self, fields: dict):
        arrs = [np.ascontiguousarray(np.broadcast_to(fields[k], self.shape), dtype=np.float64)
                for k in FIELDS]
        _check(lib().ehd_set_fields(self.h, *[_ptr(a) for a in arrs]))

    def initialize(self):
        _check(lib().ehd_initialize(self.h))

    def get_fields(self, names=FIELDS) -> dict:
        out = {k: np.empty(self.shape, np.float64) for k in names}
        ptrs = [(_ptr(out[k]) if k in out else None) for k in FIELDS]
        _check(lib().ehd_get_fields(self.h, *ptrs))
        return out

    def step(self, n: int = 1):
        _check(lib().ehd_step(self.h, int(n)))

    def step_sampled(self, n: int) -> dict:
        """Steps n >= 1 steps; the diagnostics after the last one, with nu_e
        the mean of the currents after the last two steps over I0, as
        ehd_run_to_saturation samples it (the injector makes the current
        alternate with a period of two steps)."""
        return _sampled([self], n, self.step)[0]

    def stream_collide_save(self):
        _check(lib().ehd_stream_collide_save(self.h))

    def poisson(self):
        _check(lib().ehd_poisson(self.h))

    def synchronize(self):
        _check(lib().ehd_synchronize(self.h))

    def current(self) -> float:
        c = ctypes.c_double()
        _check(lib().ehd_current(self.h, ctypes.byref(c)))
        return c.value

    def set_reference_current(self, i0: float):
        _check(lib().ehd_set_reference_current(self.h, float(i0)))

    def diagnostics(self) -> dict:
        d = Diag()
        _check(lib().ehd_diagnostics(self.h, ctypes.byref(d)))
        return d.as_dict()

    def set_state_seeded(self, profile: dict, seed: int = 0, amp: float = 1e-3):
        prof = np.ascontiguousarray(np.concatenate([np.asarray(profile[k], np.float64)
                                                    for k in FIELDS]))
        _check(lib().ehd_set_state_seeded(self.h, _ptr(prof), int(seed), float(amp)))

    def set_state_from_column(self, column: "Simulation", seed: int = 0, amp: float = 1e-3):
        """ehd_set_state_from_column: the column's state broadcast over x, y
        plus the seeded velocity perturbation."""
        _check(lib().ehd_set_state_from_column(self.h, column.h, int(seed), float(amp)))

    def run_to_saturation(self, sample_every=1000, tol=1e-3, hold=3, max_steps=10**7):
        nu = ctypes.c_double()
        steps = ctypes.c_int64()
        sat = ctypes.c_int()
        _check(lib().ehd_run_to_saturation(self.h, int(sample_every), float(tol), int(hold),
                                           int(max_steps), ctypes.byref(nu), ctypes.byref(steps),
                                           ctypes.byref(sat)))
        return {"nu_e": nu.value, "steps": steps.value, "saturated": bool(sat.value)}

    def checkpoint(self, path):
        _check(lib().ehd_checkpoint(self.h, str(path).encode()))

    def restore(self, path):
        _check(lib().ehd_restore(self.h, str(path).encode()))

    def write_data_end(self, path):
        _check(lib().ehd_write_data_end(self.h, str(path).encode()))

    def read_data_end(self, path):
        _check(lib().ehd_read_data_end(self.h, str(path).encode()))

    def write_dmd(self, path):
        _check(lib().ehd_write_dmd(self.h, str(path).encode()))

    def write_tecplot(self, path, first=True):
        _check(lib().ehd_write_tecplot(self.h, str(path).encode(), int(bool(first))))

    def get_tuning(self) -> dict:
        t = Tuning()
        _check(lib().ehd_get_tuning(self.h, ctypes.byref(t)))
        return t.as_dict()

    def set_tuning(self, **kw):
        t = Tuning()
        _check(lib().ehd_get_tuning(self.h, ctypes.byref(t)))
        for k, v in kw.items():
            setattr(t, k, int(v))
        _check(lib().ehd_set_tuning(self.h, ctypes.byref(t)))

    def device_bytes(self) -> int:
        b = ctypes.c_size_t()
        _check(lib().ehd_device_bytes(self.h, ctypes.byref(b)))
        return b.value


class Batch:
    """Independent instances on one GPU, stepped together (ehd_batch)."""

    def __init__(self, params: list, precision: str = "fp32", device: int = 0):
        arr = (Params * len(params))(*params)
        cfg = Config(precision=PRECISIONS[precision], device=device)
        h = _vp()
        _check(lib().ehd_batch_create(arr, len(params), ctypes.byref(cfg), ctypes.byref(h)))
        self.h = h
        self.params = list(params)
        self.instances = []
        for i, p in enumerate(self.params):
            c = _vp()
            _check(lib().ehd_batch_instance(self.h, i, ctypes.byref(c)))
            self.instances.append(Simulation._view(c, p))

    def __len__(self):
        return len(self.instances)

    def __getitem__(self, i) -> Simulation:
        return self.instances[i]

    def set_active(self, i: int, active: bool):
        _check(lib().ehd_batch_set_active(self.h, int(i), int(bool(active))))

    def set_mode(self, mode: int):
        """ehd_batch_set_mode: 1 per-instance graph branches (default), 0
        grouped launches."""
        _check(lib().ehd_batch_set_mode(self.h, int(mode)))

    def step(self, n: int = 1):
        _check(lib().ehd_batch_step(self.h, int(n)))

    def step_sampled(self, n: int) -> list:
        """Simulation.step_sampled for every instance: one list entry each."""
        return _sampled(self.instances, n, self.step)

    def autotune(self, trial_steps: int = 20):
        _check(lib().ehd_batch_autotune(self.h, int(trial_steps)))

    def run_to_saturation(self, sample_every=1000, tol=1e-3, hold=3, max_steps=10**7):
        n = len(self)
        sat = (ctypes.c_int32 * n)()
        steps = (ctypes.c_int64 * n)()
        nu = (ctypes.c_double * n)()
        _check(lib().ehd_batch_run_to_saturation(self.h, int(sample_every), float(tol),
                                                 int(hold), int(max_steps), sat, steps, nu))
        # saturated: True, False (budget used up) or None (a field went non-finite)
        st = {1: True, 0: False, -1: None}
        return [{"saturated": st[sat[i]], "steps": steps[i], "nu_e": nu[i]} for i in range(n)]

    def close(self):
        if getattr(self, "h", None):
            for sim in self.instances:
                sim.h = None
            lib().ehd_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
