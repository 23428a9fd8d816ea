"""Tensor-core (tcgen05) BF16 kernels of the learned warm start: GEMMs
against a PyTorch FP32 reference, MLP gradients against the CPU oracle."""
import numpy as np
import pytest

from tests.conftest import cuda_available

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="CUDA device required")]


def ops():
    from co_cultivation_metabolic_atlas_b200.warmstart import TensorCoreOps
    return TensorCoreOps()


def ref_gemm(A, B, transA, transB):
    a = A.float().t() if transA else A.float()
    b = B.float().t() if transB else B.float()
    return a @ b.t()


@pytest.mark.parametrize("M,N,K,tA,tB", [
    (128, 128, 64, False, False),     # exactly one tile, one K slice
    (128, 128, 256, False, False),    # several K slices through both stages
    (200, 300, 100, False, False),    # ragged in every dimension
    (257, 130, 520, True, False),
    (96, 77, 129, False, True),
    (300, 260, 96, True, True),
])
def test_gemm_matches_fp32_reference(M, N, K, tA, tB):
    import torch
    g = torch.Generator(device="cpu").manual_seed(M * 7 + N)
    A = (torch.randn(K, M, generator=g) if tA else torch.randn(M, K, generator=g)).cuda().bfloat16()
    B = (torch.randn(K, N, generator=g) if tB else torch.randn(N, K, generator=g)).cuda().bfloat16()
    C = torch.empty(M, N, device="cuda")
    o = ops()
    o.gemm(A, B, M, N, K, transA=tA, transB=tB, out32=C)
    torch.cuda.synchronize()
    assert o.error_flag() == 0
    ref = ref_gemm(A, B, tA, tB)
    torch.testing.assert_close(C, ref, rtol=1e-4, atol=1e-4 * K ** 0.5)


@pytest.mark.parametrize("M,N,K,tA,tB", [
    (264, 136, 72, False, False),     # TMA-fed kernel: ragged tiles, every operand storage
    (264, 136, 72, True, False),
    (264, 136, 72, False, True),
    (264, 136, 72, True, True),
    (520, 264, 4096, True, True),     # weight-gradient shape: 64 k-tiles through the stage ring
    (4096, 1024, 512, False, False),  # many tiles, two CTAs per SM
])
def test_tma_gemm_matches_fp32_reference(M, N, K, tA, tB):
    """Operands on 16-byte boundaries with row strides of multiples of 8
    elements take the TMA-fed kernel (K-major or MN-major tiles)."""
    import torch
    g = torch.Generator(device="cpu").manual_seed(M + 3 * N + K)
    A = (torch.randn(K, M, generator=g) if tA else torch.randn(M, K, generator=g)).cuda().bfloat16()
    B = (torch.randn(K, N, generator=g) if tB else torch.randn(N, K, generator=g)).cuda().bfloat16()
    C = torch.empty(M, N, device="cuda")
    o = ops()
    o.gemm(A, B, M, N, K, transA=tA, transB=tB, out32=C)
    torch.cuda.synchronize()
    assert o.error_flag() == 0
    torch.testing.assert_close(C, ref_gemm(A, B, tA, tB), rtol=1e-4, atol=1e-4 * K ** 0.5)


@pytest.mark.parametrize("pad", [0, 3])
def test_both_gemm_kernels_agree_and_accumulate(pad):
    """The same product through the TMA-fed kernel (aligned operands) and
    the register-staged one (operands shifted off the 16-byte boundary),
    accumulated into an FP32 output with an aligned or odd row stride."""
    import torch
    g = torch.Generator(device="cpu").manual_seed(11 + pad)
    M, N, K = 200, 144, 136
    A = torch.randn(M, K, generator=g).cuda().bfloat16()
    B = torch.randn(N, K, generator=g).cuda().bfloat16()
    shifted = []
    for X in (A, B):
        buf = torch.zeros(X.numel() + 8, dtype=torch.bfloat16, device="cuda")
        buf[1:1 + X.numel()] = X.reshape(-1)
        shifted.append(buf[1:1 + X.numel()].view(X.shape))
    assert shifted[0].data_ptr() % 16 != 0
    o = ops()
    base = torch.randn(M, N + pad, generator=g).cuda()
    outs = []
    for a, b in ((A, B), tuple(shifted)):
        C = base.clone()
        o.gemm(a, b, M, N, K, out32=C, accumulate=True)
        outs.append(C)
    torch.cuda.synchronize()
    assert o.error_flag() == 0
    ref = base.clone()
    ref[:, :N] += ref_gemm(A, B, False, False)
    for C in outs:
        torch.testing.assert_close(C, ref, rtol=1e-4, atol=1e-4 * K ** 0.5)
    torch.testing.assert_close(outs[0], outs[1], rtol=1e-5, atol=1e-5)


def test_gemm_bias_gelu_epilogue_and_bf16_output():
    import torch
    from co_cultivation_metabolic_atlas_b200.warmstart import EPI_BIAS_GELU
    g = torch.Generator(device="cpu").manual_seed(3)
    M, N, K = 150, 520, 48
    A = torch.randn(M, K, generator=g).cuda().bfloat16()
    B = torch.randn(N, K, generator=g).cuda().bfloat16()
    bias = torch.randn(N, generator=g).cuda()
    C16 = torch.empty(M, N, device="cuda", dtype=torch.bfloat16)
    Z = torch.empty(M, N, device="cuda")
    ops().gemm(A, B, M, N, K, bias=bias, epilogue=EPI_BIAS_GELU, out16=C16, Z=Z)
    torch.cuda.synchronize()
    zref = ref_gemm(A, B, False, False) + bias
    torch.testing.assert_close(Z, zref, rtol=1e-4, atol=1e-3)
    href = torch.nn.functional.gelu(zref)
    torch.testing.assert_close(C16.float(), href, rtol=1e-2, atol=1e-2)


def test_mlp_gradients_match_cpu_oracle():
    import torch
    from co_cultivation_metabolic_atlas_b200.warmstart import MLP
    from oracle import mlp as om
    net = MLP([44, 64, 64, 200], seed=1)
    rng = np.random.default_rng(4)
    X = torch.tensor(rng.normal(size=(96, 44)), dtype=torch.float32, device="cuda")
    T = torch.tensor(rng.normal(size=(96, 200)), dtype=torch.float32, device="cuda")
    Y = net.forward(X, keep=True)
    Tp = torch.zeros_like(Y)
    Tp[:, :200] = T
    dY = torch.empty_like(Y)
    dY16 = torch.empty(Y.shape, dtype=torch.bfloat16, device="cuda")
    net.ops.mse_grad(Y, Tp, 1.0, dY32=dY, dY16=dY16)
    gW, gb = net.backward(dY, dY16)
    torch.cuda.synchronize()
    W = [w.cpu().numpy() for w in net.W]
    b = [v.cpu().numpy() for v in net.b]
    Xp = np.zeros((96, net.pdims[0]), np.float32)
    Xp[:, :44] = X.cpu().numpy()
    Yo, cache = om.forward(W, b, Xp)
    np.testing.assert_allclose(Y.cpu().numpy(), Yo, rtol=2e-2, atol=2e-2)
    gWo, gbo = om.backward(W, cache, dY.cpu().numpy())
    for l in range(net.layers):
        a, r = gW[l].cpu().numpy(), gWo[l]
        assert np.linalg.norm(a - r) <= 2e-2 * np.linalg.norm(r) + 1e-6, l
        a, r = gb[l].cpu().numpy(), gbo[l]
        assert np.linalg.norm(a - r) <= 2e-2 * np.linalg.norm(r) + 1e-6, l


def test_training_reduces_loss_on_a_smooth_map():
    import torch
    from co_cultivation_metabolic_atlas_b200.warmstart import MLP, train
    rng = np.random.default_rng(5)
    X = torch.tensor(rng.normal(size=(8192, 44)), dtype=torch.float32, device="cuda")
    P = torch.tensor(rng.normal(size=(44, 300)) / 7.0, dtype=torch.float32, device="cuda")
    T = torch.tanh(X @ P)
    net = MLP([44, 128, 128, 300], seed=2)
    losses = train(net, X, T, epochs=8, batch=1024, lr=2e-3, lr_final=5e-4)
    assert losses[-1] < 0.25 * losses[0]
