"""The Fourier neural operator on the GPU (include/ehd_fno.h): the BF16
tensor-core product it is built on, and its forward pass and gradients against
the float64 CPU restatement (oracle/fno_oracle.py) with the same parameters.

Every contraction rounds its operands to BF16 and accumulates in FP32, so the
product is checked tightly against float64 products of the BF16-rounded
operands, and the network against float64 within the few-percent error that
BF16 operands leave after a dozen chained contractions."""
import numpy as np
import pytest

from conftest import fno
import fno_oracle as F

pytestmark = pytest.mark.gpu

SMALL = dict(nx=16, ny=12, nz=9, in_channels=4, out_channels=3, width=8, layers=3, modes_x=3,
             modes_y=2, modes_z=2, hidden=16)


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


# Kernel by case: the row-streaming one (A with unit stride along k, K in 16,
# 32, 64, 128, N <= 128) for the first four and (24, 32, 64), (1000, 32, 64),
# (16, 8, 16): partial 16-row tiles, odd C rows (single-element stores),
# batches; the small-left-matrix one (one A, M, K <= 128, B with unit stride
# along n) for (17, 9, 112) and the last four: M = 9..128, K = 5..128
# (partial K steps), odd N; the small-K one (K <= 16, N <= 128, A and C
# row-major) for the last three, shaped like the lift and the projection's
# input gradient; the tiled one for the rest (K = 200, a transposed A per
# product, K = 1000)
@pytest.mark.parametrize("M,N,K,batch,ta,tb", [(64, 64, 32, 1, False, False),
                                               (37, 5, 128, 2, False, False),
                                               (300, 128, 32, 1, False, False),
                                               (45, 17, 16, 3, False, False),
                                               (37, 91, 200, 3, False, False),
                                               (130, 70, 48, 2, True, False),
                                               (1, 5, 1000, 1, True, True),
                                               (24, 32, 64, 5, False, True),
                                               (1000, 32, 64, 1, False, True),
                                               (16, 8, 16, 1, False, False),
                                               (17, 9, 112, 1, False, False),
                                               (100, 300, 40, 1, True, False),
                                               (24, 1000, 64, 1, True, False),
                                               (128, 77, 128, 1, True, False),
                                               (9, 33, 5, 1, True, False),
                                               (5000, 32, 9, 1, False, False),
                                               (3000, 128, 5, 1, False, True),
                                               (77, 100, 3, 1, False, False)])
def test_gemm_matches_float64_products_of_bf16_operands(M, N, K, batch, ta, tb):
    import torch
    g = torch.Generator().manual_seed(M * N + K)
    A = torch.randn(batch, K, M, generator=g).cuda().transpose(1, 2) if ta else \
        torch.randn(batch, M, K, generator=g).cuda()
    B = torch.randn(batch, N, K, generator=g).cuda().transpose(1, 2) if tb else \
        torch.randn(batch, K, N, generator=g).cuda()
    C0 = torch.randn(batch, M, N, generator=g).cuda()
    C = C0.clone()
    fno.gemm(A, B, C, alpha=0.5, beta=2.0)
    ref = 0.5 * (A.bfloat16().double() @ B.bfloat16().double()) + 2.0 * C0.double()
    err = (C.double() - ref).abs().max().item() / ref.abs().max().item()
    assert err < 1e-5, err


@pytest.mark.parametrize("M,N,K,batch", [(24, 8192, 64, 16), (64, 8192, 48, 8),
                                         (128, 4096, 40, 8), (24, 1004, 64, 48),
                                         (40, 1002, 33, 48)])
def test_gemm_with_one_left_matrix_for_the_batch(M, N, K, batch):
    """The small-left-matrix kernel with 32-, 16- and 8-column warp units (it
    takes the widest that still leaves 4096 units): one A for every product
    of the batch, as the truncated DFTs have it.  B's rows are 16-byte
    aligned (N a multiple of 4: B staged by asynchronous copies, partial last
    units zero-filled) or not (N = 1002: fragments loaded from global
    memory)."""
    import torch
    g = torch.Generator().manual_seed(M + N + K)
    A = torch.randn(1, M, K, generator=g).cuda().expand(batch, M, K)
    B = torch.randn(batch, K, N, generator=g).cuda()
    C0 = torch.randn(batch, M, N, generator=g).cuda()
    C = C0.clone()
    fno.gemm(A, B, C, alpha=0.5, beta=2.0)
    ref = 0.5 * (A.bfloat16().double() @ B.bfloat16().double()) + 2.0 * C0.double()
    err = (C.double() - ref).abs().max().item() / ref.abs().max().item()
    assert err < 1e-5, err


# width 16, hidden 32: the pointwise layers, the projection and their input
# gradients run on the row-streaming kernel (bias, GELU second output)
WIDE = dict(SMALL, width=16, hidden=32)


def make(seed=3, max_batch=2, cfg=SMALL):
    return fno.FNO(cfg["nx"], cfg["ny"], cfg["nz"], cfg["in_channels"],
                   cfg["out_channels"], width=cfg["width"], layers=cfg["layers"],
                   modes=(cfg["modes_x"], cfg["modes_y"], cfg["modes_z"]),
                   hidden=cfg["hidden"], max_batch=max_batch, seed=seed)


def data(seed, batch=2, cfg=SMALL):
    rng = np.random.default_rng(seed)
    sh = (batch, cfg["nz"], cfg["ny"], cfg["nx"])
    a = rng.standard_normal(sh + (cfg["in_channels"],)).astype(np.float32)
    t = rng.standard_normal(sh + (SMALL["out_channels"],)).astype(np.float32)
    return a, t


@pytest.mark.parametrize("cfg", [SMALL, WIDE], ids=["width8", "width16"])
def test_forward_and_gradients_match_the_oracle(cfg):
    import torch
    a, t = data(1, cfg=cfg)
    with make(cfg=cfg) as net:
        p = net.params()
        # larger spectral weights than the initialisation, so that the
        # spectral path carries a share of the output comparable to the rest
        rng = np.random.default_rng(2)
        p = (p + 0.05 * rng.standard_normal(p.size)).astype(np.float32)
        net.set_params(p)
        u = net.forward(torch.tensor(a).cuda()).cpu().numpy()
        loss = net.backward(torch.tensor(a).cuda(), torch.tensor(t).cuda())
        g = net.grads()
    lref, gref, uref = F.loss_and_grads(p, a, t, cfg)
    assert rel(u, uref) < 2e-2, rel(u, uref)
    assert loss == pytest.approx(lref, rel=2e-2)
    assert rel(g, gref) < 5e-2, rel(g, gref)
    cos = float(g @ gref / np.linalg.norm(g) / np.linalg.norm(gref))
    assert cos > 0.998, cos


def test_adam_training_fits_a_teacher_network():
    """A student with its own initialisation learns the map of a teacher
    network of the same shape: the loss falls by an order of magnitude."""
    import torch
    a, _ = data(5)
    a = torch.tensor(a).cuda()
    with make(seed=9) as teacher:
        p = teacher.params()
        teacher.set_params(p + 0.05 * np.random.default_rng(3).standard_normal(p.size))
        t = teacher.forward(a)
    with make(seed=4) as net:
        first = net.backward(a, t)
        for _ in range(300):
            net.backward(a, t)
            net.adam_step(lr=3e-3)
        last = net.backward(a, t)
    assert last < 0.1 * first, (first, last)
