"""Accuracy of the split-y slab kernel's z solve, restated in numpy.

The slab kernel (ehd-convection-3d_b200/csrc/poisson.cu, poisson_slab) solves
per (kx, ky) mode the system of the reference's odd-extension transform
(poisson.cu:78-167), x(z-1) - beta x(z) + x(z+1) = d(z) on the n = NZ - 2
interior planes with x = 0 on the electrodes, beta = 2 + h, from both ends at
once: the planes 0..m-1 are eliminated downwards and n-1..n-m upwards with the
same pivots c_0..c_{m-1} (the matrix is symmetric Toeplitz), the middle plane m
takes mu = 1/(-beta - 2 c_{m-1}), and each half is substituted back.  Pivots
and mu are built in FP64 and stored in FP32; the arithmetic is FP64, and the
eliminated rows and the solution are stored in FP32 between the sweeps, as in
the kernel's shared-memory slab.

Checked against a dense FP64 solve, over the interior-plane counts of the
kernel's sizes (NZ = 33, 65, 129, 257) and the range of h of the bench and
fine grids (h = (kx^2 + ky^2) dz^2 from 1.5e-4 up).
"""
import numpy as np
import pytest


def pivots(h, m):
    beta = 2.0 + h
    c, prev = np.zeros(m), 0.0
    for i in range(m):
        prev = 1.0 / (-beta - prev)
        c[i] = prev
    return c, 1.0 / (-beta - 2.0 * c[-1])


def two_sided(h, d):
    """The kernel's order of operations: FP32 tables, FP64 arithmetic, FP32
    storage of the eliminated rows and of the result."""
    n = len(d)
    m = (n - 1) // 2
    c, mu = pivots(h, m)
    c = c.astype(np.float32).astype(np.float64)
    mu = float(np.float32(mu))
    d = d.astype(np.float32).astype(np.float64)
    top, bot = np.zeros(m, np.float32), np.zeros(m, np.float32)
    a = b = 0.0
    for k in range(m):
        a = (d[k] - a) * c[k]
        b = (d[n - 1 - k] - b) * c[k]
        top[k], bot[k] = a, b
    x = np.zeros(n, np.float32)
    xm = (d[m] - a - b) * mu
    x[m] = xm
    xa = xb = xm
    for k in range(m - 1, -1, -1):
        xa = float(top[k]) - c[k] * xa
        xb = float(bot[k]) - c[k] * xb
        x[k], x[n - 1 - k] = xa, xb
    return x.astype(np.float64)


def dense(h, d):
    n = len(d)
    A = (np.diag(np.full(n, -(2.0 + h))) + np.diag(np.ones(n - 1), 1)
         + np.diag(np.ones(n - 1), -1))
    return np.linalg.solve(A, d)


@pytest.mark.parametrize("n", [31, 63, 127, 255])
@pytest.mark.parametrize("h", [1.5e-4, 6e-4, 1e-2, 0.3, 20.0])
def test_two_sided_thomas_matches_dense_solve(n, h):
    rng = np.random.default_rng(n)
    z = np.linspace(0.0, 1.0, n + 2)[1:-1]
    worst = 0.0
    for d in (np.exp(-3.0 * z) * (1.0 + 0.1 * np.sin(7.0 * z)), rng.standard_normal(n),
              np.exp(-3.0 * z) * rng.standard_normal(n)):
        d = d.astype(np.float32).astype(np.float64)
        ref = dense(h, d)
        worst = max(worst, np.max(np.abs(two_sided(h, d) - ref)) / np.max(np.abs(ref)))
    # FP32 storage of the result alone is 6e-8; the elimination adds the rest
    assert worst < 6e-7, worst


def test_middle_plane_closes_the_two_halves():
    """In exact arithmetic the two-sided solve is the solution: FP64 tables and
    storage reproduce the dense solve to round-off."""
    n, h = 127, 6e-4
    d = np.random.default_rng(1).standard_normal(n)
    m = (n - 1) // 2
    c, mu = pivots(h, m)
    a = b = 0.0
    top, bot = np.zeros(m), np.zeros(m)
    for k in range(m):
        a = (d[k] - a) * c[k]
        b = (d[n - 1 - k] - b) * c[k]
        top[k], bot[k] = a, b
    x = np.zeros(n)
    x[m] = (d[m] - a - b) * mu
    xa = xb = x[m]
    for k in range(m - 1, -1, -1):
        xa = top[k] - c[k] * xa
        xb = bot[k] - c[k] * xb
        x[k], x[n - 1 - k] = xa, xb
    ref = dense(h, d)
    assert np.max(np.abs(x - ref)) / np.max(np.abs(ref)) < 1e-11
