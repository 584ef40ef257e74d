"""ctypes binding of include/ehd_fno.h: the Fourier neural operator warm start.

Tensors cross the boundary as CUDA device pointers; torch tensors are the
container here (channels-last FP32, [batch][z][y][x][channel]).
"""
from __future__ import annotations

import ctypes

import numpy as np

import ehd

_i = ctypes.c_int
_vp = ctypes.c_void_p
_fp = ctypes.POINTER(ctypes.c_float)
_i64 = ctypes.c_int64


class Config(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("nz", ctypes.c_int32),
                ("in_channels", ctypes.c_int32), ("out_channels", ctypes.c_int32),
                ("width", ctypes.c_int32), ("layers", ctypes.c_int32),
                ("modes_x", ctypes.c_int32), ("modes_y", ctypes.c_int32),
                ("modes_z", ctypes.c_int32), ("hidden", ctypes.c_int32),
                ("max_batch", ctypes.c_int32), ("seed", ctypes.c_uint64),
                ("device", ctypes.c_int32), ("reserved", ctypes.c_int32 * 5)]


# every symbol include/ehd_fno.h declares, with (restype, argtypes)
SIGNATURES = {
    "ehd_fno_create": (_i, [ctypes.POINTER(Config), ctypes.POINTER(_vp)]),
    "ehd_fno_destroy": (_i, [_vp]),
    "ehd_fno_param_count": (_i, [_vp, ctypes.POINTER(_i64)]),
    "ehd_fno_get_params": (_i, [_vp, _fp]),
    "ehd_fno_set_params": (_i, [_vp, _fp]),
    "ehd_fno_forward": (_i, [_vp, _i, _vp, _vp]),
    "ehd_fno_backward": (_i, [_vp, _i, _vp, _vp, ctypes.POINTER(ctypes.c_double)]),
    "ehd_fno_get_grads": (_i, [_vp, _fp]),
    "ehd_fno_adam_step": (_i, [_vp, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                               ctypes.c_float]),
    "ehd_fno_synchronize": (_i, [_vp]),
    "ehd_bf16_gemm": (_i, [_i, _i, _i, _i, _vp, _i64, _i64, _i64, _vp, _i64, _i64, _i64, _vp,
                           _i64, _i64, _i64, ctypes.c_float, ctypes.c_float, _vp]),
}

_lib = None


def lib():
    """libehd.so through a handle of this module's own, so that the argument
    types bound here (this module's Config) do not clash with another copy of
    this module loaded under a different name."""
    global _lib
    if _lib is None:
        ehd.lib()  # raises if the library was not built
        L = ctypes.CDLL(str(ehd.LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _fptr(a: np.ndarray):
    return a.ctypes.data_as(_fp)


def gemm(A, B, C, alpha=1.0, beta=0.0):
    """C[b] = alpha A[b] @ B[b] + beta C[b] on the BF16 tensor cores, for
    3-D CUDA float32 tensors (any strides)."""
    bt, M, K = A.shape
    _, _, N = B.shape
    ehd._check(lib().ehd_bf16_gemm(M, N, K, bt, A.data_ptr(), A.stride(1), A.stride(2),
                                   A.stride(0), B.data_ptr(), B.stride(1), B.stride(2),
                                   B.stride(0), C.data_ptr(), C.stride(1), C.stride(2),
                                   C.stride(0), float(alpha), float(beta), None))


class FNO:
    """One Fourier neural operator (ehd_fno) on one GPU."""

    def __init__(self, nx, ny, nz, in_channels, out_channels, width=32, layers=4, modes=(12, 12, 12),
                 hidden=128, max_batch=4, seed=0, device=0):
        self.cfg = Config(nx=nx, ny=ny, nz=nz, in_channels=in_channels,
                          out_channels=out_channels, width=width, layers=layers,
                          modes_x=modes[0], modes_y=modes[1], modes_z=modes[2], hidden=hidden,
                          max_batch=max_batch, seed=seed, device=device)
        h = _vp()
        ehd._check(lib().ehd_fno_create(ctypes.byref(self.cfg), ctypes.byref(h)))
        self.h = h
        n = _i64()
        ehd._check(lib().ehd_fno_param_count(self.h, ctypes.byref(n)))
        self.nparam = n.value

    def close(self):
        if getattr(self, "h", None):
            lib().ehd_fno_destroy(self.h)
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

    def params(self) -> np.ndarray:
        out = np.empty(self.nparam, np.float32)
        ehd._check(lib().ehd_fno_get_params(self.h, _fptr(out)))
        return out

    def set_params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        assert p.size == self.nparam
        ehd._check(lib().ehd_fno_set_params(self.h, _fptr(p)))

    def grads(self) -> np.ndarray:
        out = np.empty(self.nparam, np.float32)
        ehd._check(lib().ehd_fno_get_grads(self.h, _fptr(out)))
        return out

    def forward(self, a):
        """a: CUDA float32 [batch, nz, ny, nx, in_channels] -> u of out_channels."""
        import torch
        a = a.contiguous()
        u = torch.empty(a.shape[:-1] + (self.cfg.out_channels,), dtype=torch.float32,
                        device=a.device)
        ehd._check(lib().ehd_fno_forward(self.h, a.shape[0], a.data_ptr(), u.data_ptr()))
        self.synchronize()
        return u

    def backward(self, a, target) -> float:
        a, target = a.contiguous(), target.contiguous()
        loss = ctypes.c_double()
        ehd._check(lib().ehd_fno_backward(self.h, a.shape[0], a.data_ptr(), target.data_ptr(),
                                          ctypes.byref(loss)))
        return loss.value

    def adam_step(self, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8):
        ehd._check(lib().ehd_fno_adam_step(self.h, lr, beta1, beta2, eps))

    def synchronize(self):
        ehd._check(lib().ehd_fno_synchronize(self.h))


def main(argv=None):
    """Times the network's forward pass and training step (backward + Adam)
    on random inputs of the given grid and batch: wall time over `steps`
    calls between two synchronisations of the network's stream.

        python ehd-convection-3d_b200/fno.py --grid 64 64 33 --batch 4
    """
    import argparse
    import json
    import time

    import torch
    ap = argparse.ArgumentParser(description="time the FNO forward pass and training step")
    ap.add_argument("--grid", type=int, nargs=3, default=(64, 64, 33), metavar=("NX", "NY", "NZ"))
    ap.add_argument("--in-channels", type=int, default=9)
    ap.add_argument("--out-channels", type=int, default=5)
    ap.add_argument("--width", type=int, default=32)
    ap.add_argument("--layers", type=int, default=4)
    ap.add_argument("--modes", type=int, default=12)
    ap.add_argument("--hidden", type=int, default=128)
    ap.add_argument("--batch", type=int, default=4)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    a = ap.parse_args(argv)
    nx, ny, nz = a.grid
    net = FNO(nx, ny, nz, a.in_channels, a.out_channels, width=a.width, layers=a.layers,
              modes=(a.modes, a.modes, min(a.modes, nz // 2)), hidden=a.hidden,
              max_batch=a.batch, seed=7)
    g = torch.Generator(device="cuda").manual_seed(0)
    x = torch.randn(a.batch, nz, ny, nx, a.in_channels, device="cuda", generator=g)
    t = torch.randn(a.batch, nz, ny, nx, a.out_channels, device="cuda", generator=g)
    for _ in range(a.warmup):
        net.forward(x)
        net.backward(x, t)
        net.adam_step(1e-4)
    net.synchronize()
    t0 = time.perf_counter()
    for _ in range(a.steps):
        net.forward(x)
    net.synchronize()
    t1 = time.perf_counter()
    for _ in range(a.steps):
        net.backward(x, t)
        net.adam_step(1e-4)
    net.synchronize()
    t2 = time.perf_counter()
    out = {"grid": [nx, ny, nz], "batch": a.batch, "width": a.width, "layers": a.layers,
           "modes": a.modes, "parameters": net.nparam,
           "forward_ms": 1e3 * (t1 - t0) / max(1, a.steps),
           "train_step_ms": 1e3 * (t2 - t1) / max(1, a.steps)}
    print(json.dumps(out), flush=True)
    net.close()
    return out


if __name__ == "__main__":
    main()
