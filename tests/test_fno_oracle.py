"""The CPU restatement of the Fourier neural operator (oracle/fno_oracle.py):
its spectral convolution against the defining sums, written out with explicit
loops over the kept modes (CPU only)."""
import numpy as np

from conftest import ROOT  # noqa: F401  (puts oracle/ on the path)
import fno_oracle as F


def test_spectral_convolution_equals_the_defining_sums():
    c = dict(modes_x=2, modes_y=1, modes_z=1)
    rng = np.random.default_rng(0)
    B, Z, Y, X, W = 1, 4, 3, 6, 2
    v = rng.standard_normal((B, Z, Y, X, W))
    modes = 2 * 2 * 2
    Rre = rng.standard_normal((modes, W, W))
    Rim = rng.standard_normal((modes, W, W))
    import torch
    got = F.spectral(torch.tensor(v), torch.tensor(Rre), torch.tensor(Rim), c).numpy()
    ky = [F.wave(j, 1, Y) for j in range(2)]
    kz = [F.wave(j, 1, Z) for j in range(2)]
    zz, yy, xx = np.meshgrid(np.arange(Z), np.arange(Y), np.arange(X), indexing="ij")
    want = np.zeros((Z, Y, X, W))
    m = 0
    for a in kz:
        for b in ky:
            for k in range(2):
                ph = np.exp(-2j * np.pi * (a * zz / Z + b * yy / Y + k * xx / X))
                vhat = np.array([(v[0, ..., i] * ph).sum() for i in range(W)])
                out = (Rre[m] + 1j * Rim[m]) @ vhat
                weight = 1.0 if k == 0 else 2.0  # the real inverse along x
                for o in range(W):
                    want[..., o] += weight * np.real(out[o] * np.conj(ph)) / (X * Y * Z)
                m += 1
    assert np.abs(got[0] - want).max() < 1e-12 * np.abs(want).max()


def test_loss_gradient_matches_finite_differences():
    c = dict(nx=6, ny=4, nz=4, in_channels=2, out_channels=1, width=3, layers=2, modes_x=2,
             modes_y=1, modes_z=1, hidden=4)
    modes = 2 * 2 * 2
    n = 2 * 3 + 3 + 2 * (9 + 3 + 2 * modes * 9) + 3 * 4 + 4 + 4 + 1
    rng = np.random.default_rng(1)
    p = 0.3 * rng.standard_normal(n)
    a = rng.standard_normal((1, 4, 4, 6, 2))
    t = rng.standard_normal((1, 4, 4, 6, 1))
    loss, g, _ = F.loss_and_grads(p, a, t, c)
    for i in rng.choice(n, 12, replace=False):
        e = np.zeros(n)
        e[i] = 1e-6
        num = (F.loss_and_grads(p + e, a, t, c)[0] - F.loss_and_grads(p - e, a, t, c)[0]) / 2e-6
        assert abs(num - g[i]) < 1e-6 + 1e-5 * abs(num), (i, num, g[i])
