"""CPU restatement of the Fourier neural operator of include/ehd_fno.h, in
float64 with torch.fft and autograd -- the checker of the GPU forward pass and
its gradients.  Test infrastructure only.

The operator is the published Fourier neural operator (Li et al., "Fourier
Neural Operator for Parametric Partial Differential Equations", 2021):
lift, Fourier layers v <- gelu(K(v) + v W + b) (no activation after the last),
projection gelu(v Q1 + q1) Q2 + q2, with K(v) = irfft_x ifft_y ifft_z of
R . (truncated fft_z fft_y rfft_x of v).  Parameters come as the flat FP32
vector of ehd_fno_get_params, in the order that header documents.
"""
from __future__ import annotations

import numpy as np
import torch


def wave(j, m, n):
    return j if j < m else n - 2 * m + j


def unpack(p, c):
    """dict of float64 tensors from the flat parameter vector; c: config dict."""
    p = torch.as_tensor(np.asarray(p, np.float64))
    W, H, cin, cout = c["width"], c["hidden"], c["in_channels"], c["out_channels"]
    modes = 2 * c["modes_z"] * 2 * c["modes_y"] * c["modes_x"]
    out, o = {}, 0

    def take(name, *shape):
        nonlocal o
        n = int(np.prod(shape))
        out[name] = p[o:o + n].reshape(*shape).clone()
        o += n

    take("P", cin, W)
    take("p", W)
    for l in range(c["layers"]):
        take(f"W{l}", W, W)
        take(f"b{l}", W)
        take(f"Rre{l}", modes, W, W)
        take(f"Rim{l}", modes, W, W)
    take("Q1", W, H)
    take("q1", H)
    take("Q2", H, cout)
    take("q2", cout)
    assert o == p.numel()
    return out


def pack(t, c):
    names = ["P", "p"]
    for l in range(c["layers"]):
        names += [f"W{l}", f"b{l}", f"Rre{l}", f"Rim{l}"]
    names += ["Q1", "q1", "Q2", "q2"]
    return torch.cat([t[n].reshape(-1) for n in names])


def spectral(v, Rre, Rim, c):
    """v: [B, Z, Y, X, W] -> K(v), same shape."""
    B, Z, Y, X, W = v.shape
    mx, my, mz = c["modes_x"], c["modes_y"], c["modes_z"]
    ky = [wave(j, my, Y) for j in range(2 * my)]
    kz = [wave(j, mz, Z) for j in range(2 * mz)]
    vc = v.permute(0, 4, 1, 2, 3)                      # [B, W, Z, Y, X]
    s = torch.fft.rfft(vc, dim=-1)[..., :mx]
    s = torch.fft.fft(s, dim=-2)[..., ky, :]
    s = torch.fft.fft(s, dim=-3)[:, :, kz]              # [B, W, 2mz, 2my, mx]
    s = s.reshape(B, W, -1)                             # modes (kz, ky, kx)
    R = torch.complex(Rre, Rim)                         # [modes, out, in]
    o = torch.einsum("moi,bim->bom", R, s).reshape(B, W, 2 * mz, 2 * my, mx)
    full = torch.zeros(B, W, Z, Y, X // 2 + 1, dtype=o.dtype)
    idx_z = torch.tensor(kz)[:, None]
    idx_y = torch.tensor(ky)[None, :]
    full[:, :, idx_z, idx_y, :mx] = o
    r = torch.fft.ifft(torch.fft.ifft(full, dim=-3), dim=-2)
    r = torch.fft.irfft(r, n=X, dim=-1)
    return r.permute(0, 2, 3, 4, 1)


def forward(a, t, c):
    gelu = torch.nn.functional.gelu
    v = a @ t["P"] + t["p"]
    L = c["layers"]
    for l in range(L):
        z = v @ t[f"W{l}"] + t[f"b{l}"] + spectral(v, t[f"Rre{l}"], t[f"Rim{l}"], c)
        v = gelu(z) if l < L - 1 else z
    return gelu(v @ t["Q1"] + t["q1"]) @ t["Q2"] + t["q2"]


def loss_and_grads(p, a, target, c):
    """MSE loss and its gradient with respect to the flat parameters."""
    t = unpack(p, c)
    for v in t.values():
        v.requires_grad_(True)
    a = torch.as_tensor(np.asarray(a, np.float64))
    u = forward(a, t, c)
    loss = torch.mean((u - torch.as_tensor(np.asarray(target, np.float64))) ** 2)
    loss.backward()
    g = pack({k: v.grad for k, v in t.items()}, c)
    return float(loss.detach()), g.numpy(), u.detach().numpy()
