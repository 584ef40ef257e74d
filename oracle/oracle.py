"""ctypes binding of the CPU FP64 oracle (oracle/ehd_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, by ``__graft_entry__.smoke()``
as the checker, and by ``bench.py`` for the timed CPU baseline.  The product
library never loads it.

Besides the binding, this module holds the oracle-side set-up helpers that
build identical inputs for the oracle and for the product:

* ``params_from_groups`` -- the inverse of the reference's
  ``compute_parameters`` (LBM.cu:1356-1379): dimensionless T, M, C, Fe to
  mobility K, viscosity nu, injected charge q0 and diffusivity D, with
  eps, V, rho0 and Lz kept at the reference values (LBM.h:42,54-57).
* ``hydrostatic_profile`` -- the u = 0 steady state of the same discrete step,
  obtained by running the oracle on a 1 x 1 x NZ column.
* ``seeded_velocity`` -- a counter-based splitmix64 perturbation.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "libehd_oracle.so"

FIELDS = ("rho", "u", "v", "w", "q", "phi", "ex", "ey", "ez")


class Params(ctypes.Structure):
    """Mirror of ``ehd_params`` in include/ehd.h (and orc_params)."""

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


def reference_default_params(nx=122, ny=122, nz=101, **over) -> Params:
    """The reference's compiled-in constants (LBM.h:34-80) for a grid of
    nx x ny x nz nodes with dx = dy = dz = Lz/(nz-1), Lx = nx*dx, Ly = ny*dy."""
    dz = 1.0 / (nz - 1)
    p = Params(nx=nx, ny=ny, nz=nz, pad_=0,
               lx=nx * dz, ly=ny * dz, lz=1.0, dx=dz, dy=dz, dz=dz,
               dt=0.01 * dz, cfl=0.01, rho0=1600.0, charge0=10.0, voltage=1.0e4,
               eps=1.0e-4, diffu=6.25e-5, nu=0.0251004, K=2.5e-5, uw=0.0, exf=0.0,
               lambda_f=1.0 / 12.0, lambda_g=1.0e-6)
    for k, v in over.items():
        setattr(p, k, v)
    return p


def params_from_groups(nx, ny, nz, lx, ly, T, M, C, Fe, lambda_f=0.25, lambda_g=0.25,
                       cfl=0.01, **over) -> Params:
    """Inverse of compute_parameters (LBM.cu:1375-1378):
    M = sqrt(eps/rho0)/K, T = eps V/(K nu rho0), C = q0 Lz^2/(V eps), Fe = K V/D."""
    eps, V, rho0, Lz = 1.0e-4, 1.0e4, 1600.0, 1.0
    K = np.sqrt(eps / rho0) / M
    nu = eps * V / (K * T * rho0)
    q0 = C * V * eps / Lz ** 2
    D = K * V / Fe
    dz = Lz / (nz - 1)
    p = Params(nx=nx, ny=ny, nz=nz, pad_=0, lx=lx, ly=ly, lz=Lz,
               dx=lx / nx, dy=ly / ny, dz=dz, dt=cfl * dz, cfl=cfl, rho0=rho0,
               charge0=q0, voltage=V, eps=eps, diffu=D, nu=nu, K=K, uw=0.0, exf=0.0,
               lambda_f=lambda_f, lambda_g=lambda_g)
    for k, v in over.items():
        setattr(p, k, v)
    return p


def groups_of(p: Params):
    """compute_parameters, LBM.cu:1356-1379."""
    return dict(M=np.sqrt(p.eps / p.rho0) / p.K, T=p.eps * p.voltage / p.K / p.nu / p.rho0,
                C=p.charge0 * p.lz * p.lz / (p.voltage * p.eps), Fe=p.K * p.voltage / p.diffu)


_lib = None


def build():
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        L = ctypes.CDLL(str(LIB_PATH))
        dp = ctypes.POINTER(ctypes.c_double)
        L.orc_create.restype = ctypes.c_void_p
        L.orc_create.argtypes = [ctypes.POINTER(Params)]
        L.orc_destroy.argtypes = [ctypes.c_void_p]
        L.orc_set_fields.argtypes = [ctypes.c_void_p] + [dp] * 9
        L.orc_get_fields.argtypes = [ctypes.c_void_p] + [dp] * 9
        L.orc_get_pops.argtypes = [ctypes.c_void_p] + [dp] * 4
        L.orc_set_pops.argtypes = [ctypes.c_void_p] + [dp] * 4
        L.orc_step.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.orc_step_lbm.argtypes = [ctypes.c_void_p]
        L.orc_poisson.argtypes = [ctypes.c_void_p]
        L.orc_efield.argtypes = [ctypes.c_void_p]
        L.orc_init_equilibrium.argtypes = [ctypes.c_void_p]
        L.orc_initialization.argtypes = [ctypes.c_void_p]
        L.orc_current.restype = ctypes.c_double
        L.orc_current.argtypes = [ctypes.c_void_p]
        L.orc_fft1d.argtypes = [dp, ctypes.c_int, ctypes.c_int]
        L.orc_collide_only.argtypes = [ctypes.c_void_p]
        L.orc_get_post.argtypes = [ctypes.c_void_p] + [dp] * 4
        L.orc_set_threads.argtypes = [ctypes.c_int]
        L.orc_get_threads.restype = ctypes.c_int
        _lib = L
    return _lib


def _ptr(a):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def set_threads(n: int):
    lib().orc_set_threads(int(n))


def get_threads() -> int:
    return int(lib().orc_get_threads())


def fft1d(x: np.ndarray, sign: int) -> np.ndarray:
    a = np.empty(2 * len(x), np.float64)
    a[0::2] = x.real
    a[1::2] = x.imag
    lib().orc_fft1d(_ptr(a), len(x), sign)
    return a[0::2] + 1j * a[1::2]


class Oracle:
    """One simulation instance on the host, FP64, reference layout."""

    def __init__(self, p: Params):
        self.p = p
        self.shape = (p.nz, p.ny, p.nx)
        self.h = lib().orc_create(ctypes.byref(p))
        if not self.h:
            raise MemoryError("orc_create failed")

    def close(self):
        if self.h:
            lib().orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_fields(self, fields: dict):
        arrs = [np.ascontiguousarray(np.broadcast_to(fields[k], self.shape), np.float64)
                for k in FIELDS]
        lib().orc_set_fields(self.h, *[_ptr(a) for a in arrs])

    def get_fields(self) -> dict:
        out = {k: np.empty(self.shape, np.float64) for k in FIELDS}
        lib().orc_get_fields(self.h, *[_ptr(out[k]) for k in FIELDS])
        return out

    def get_pops(self):
        n = self.shape
        f0 = np.empty(n); h0 = np.empty(n)
        f1 = np.empty((26,) + n); h1 = np.empty((26,) + n)
        lib().orc_get_pops(self.h, _ptr(f0), _ptr(f1), _ptr(h0), _ptr(h1))
        return f0, f1, h0, h1

    def set_pops(self, f0, f1, h0, h1):
        a = [np.ascontiguousarray(x, np.float64) for x in (f0, f1, h0, h1)]
        lib().orc_set_pops(self.h, *[_ptr(x) for x in a])

    def collide_only(self):
        lib().orc_collide_only(self.h)

    def get_post(self):
        n = self.shape
        f0 = np.empty(n); h0 = np.empty(n)
        f2 = np.empty((26,) + n); h2 = np.empty((26,) + n)
        lib().orc_get_post(self.h, _ptr(f0), _ptr(f2), _ptr(h0), _ptr(h2))
        return f0, f2, h0, h2

    def initialization(self):
        lib().orc_initialization(self.h)

    def step(self, n: int = 1):
        lib().orc_step(self.h, int(n))

    def step_lbm(self):
        lib().orc_step_lbm(self.h)

    def poisson(self):
        lib().orc_poisson(self.h)

    def efield(self):
        lib().orc_efield(self.h)

    def current(self) -> float:
        return float(lib().orc_current(self.h))


# --------------------------------------------------------------------------
# seeded inputs
# --------------------------------------------------------------------------

_M64 = (1 << 64) - 1


def splitmix64(x: np.ndarray) -> np.ndarray:
    """splitmix64 finaliser on uint64 counters (Steele, Lea, Flood 2014)."""
    z = (x + np.uint64(0x9E3779B97F4A7C15)) & np.uint64(_M64)
    z = ((z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)) & np.uint64(_M64)
    z = ((z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)) & np.uint64(_M64)
    return z ^ (z >> np.uint64(31))


def seeded_velocity(shape, seed: int, amp: float):
    """u, v, w = amp * U(-1, 1) per node from counter-based splitmix64:
    component c of node i (linear [z][y][x] index) uses counter
    seed * 2^32 + 3 i + c.  Wall planes z = 0 and z = nz-1 are left at rest."""
    n = int(np.prod(shape))
    with np.errstate(over="ignore"):
        base = np.uint64((seed << 32) & _M64)
        idx = np.arange(n, dtype=np.uint64) * np.uint64(3) + base
        out = []
        for c in range(3):
            h = splitmix64(idx + np.uint64(c))
            r = (h >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)
            a = (amp * (2.0 * r - 1.0)).reshape(shape)
            a[0] = 0.0
            a[-1] = 0.0
            out.append(a)
    return out


def hydrostatic_profile(p: Params, tol: float = 1e-10, check_every: int = 2000,
                        max_steps: int = 2_000_000):
    """u = 0 steady state of the same discrete step on a 1 x 1 x NZ column,
    started from the reference's initialization (LBM.cu:81-96).  Returns the
    per-z profiles of all nine fields and the number of steps taken.  The run
    stops when the largest change of q, rho and phi over `check_every` steps,
    relative to each field's range, drops below `tol`."""
    q = Params(**{k: getattr(p, k) for k, _ in Params._fields_})
    q.nx = 1
    q.ny = 1
    q.lx = p.dx
    q.ly = p.dy
    o = Oracle(q)
    o.initialization()
    prev = None
    steps = 0
    while steps < max_steps:
        o.step(check_every)
        steps += check_every
        f = o.get_fields()
        cur = np.concatenate([f["q"].ravel() / max(p.charge0, 1e-300),
                              f["rho"].ravel() / p.rho0,
                              f["phi"].ravel() / p.voltage])
        if prev is not None and np.max(np.abs(cur - prev)) < tol:
            break
        prev = cur
    f = o.get_fields()
    o.close()
    return {k: f[k].reshape(-1).copy() for k in FIELDS}, steps


def state_from_profile(p: Params, prof: dict, seed: int | None = 0, amp: float = 1e-3):
    """3D fields: the per-z profile broadcast over x, y plus the seeded
    velocity perturbation (interior planes only)."""
    shape = (p.nz, p.ny, p.nx)
    f = {k: np.ascontiguousarray(np.broadcast_to(prof[k][:, None, None], shape)).copy()
         for k in FIELDS}
    if seed is not None and amp != 0.0:
        du, dv, dw = seeded_velocity(shape, seed, amp)
        f["u"] += du
        f["v"] += dv
        f["w"] += dw
    return f


def current_of(p: Params, q: np.ndarray, ez: np.ndarray) -> float:
    """current(), LBM.cu:1647-1671, on [z][y][x] arrays."""
    qt = 2.0 * q[-2] - q[-3]
    return float(np.sum(qt * ez[-1]) * p.K * p.dy * p.dy)


def data_end_view(fields: dict) -> dict:
    """The field values as the reference's save_data_end writes them
    (LBM.cu:1531-1544): rho, q, u, v, w at z = 0 and z = nz-1 replaced by a
    linear extrapolation from the two planes inside."""
    out = {k: np.array(v, copy=True) for k, v in fields.items()}
    for k in ("rho", "q", "u", "v", "w"):
        a = out[k]
        a[0] = 2.0 * a[1] - a[2]
        a[-1] = 2.0 * a[-2] - a[-3]
    return out
