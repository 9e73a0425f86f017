"""The tensor-core BF16 GEMM of the learned preconditioner (tcgen05.mma with a
TMEM accumulator and TMA operand loads), called through the C ABI, against a
torch FP32 product of the same BF16 operands. FP32 outputs agree to 1e-4 of
the largest entry (the two sum the K products in different orders); BF16
outputs to one BF16 rounding (2^-8 relative) of the largest entry."""
import pytest
import torch

import iceicle_b200 as ib

pytestmark = pytest.mark.gpu


def _ops(M, N, K, seed):
    g = torch.Generator("cuda").manual_seed(seed)
    A = torch.randn(M, K, device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, device="cuda", generator=g).to(torch.bfloat16)
    bias = torch.randn(N, device="cuda", generator=g)
    return A, B, bias


SHAPES = [(300, 256, 1296), (130, 1296, 256), (65, 100, 72), (512, 512, 64), (1, 8, 8), (257, 129, 520)]


@pytest.mark.parametrize("M,N,K", SHAPES, ids=[f"{m}x{n}x{k}" for m, n, k in SHAPES])
def test_gemm_fp32_out(M, N, K):
    A, B, _ = _ops(M, N, K, 1)
    C = torch.full((M, N), float("nan"), device="cuda")
    ib.gemm_bf16_nt(A, B, out32=C)
    ref = A.float() @ B.float().T
    assert torch.isfinite(C).all()
    assert float((C - ref).abs().max()) <= 1e-4 * float(ref.abs().max())


@pytest.mark.parametrize("M,N,K", SHAPES[:4], ids=[f"{m}x{n}x{k}" for m, n, k in SHAPES[:4]])
def test_gemm_bias_relu_bf16_out(M, N, K):
    A, B, bias = _ops(M, N, K, 2)
    C16 = torch.zeros((M, N), device="cuda", dtype=torch.bfloat16)
    C32 = torch.zeros((M, N), device="cuda")
    ib.gemm_bf16_nt(A, B, bias=bias, relu=True, out32=C32, out16=C16)
    ref = torch.relu(A.float() @ B.float().T + bias)
    scale = float(ref.abs().max())
    assert float((C32 - ref).abs().max()) <= 1e-4 * scale
    assert float((C16.float() - ref).abs().max()) <= 2.0 ** -8 * scale


def test_gemm_split_k_accumulate():
    """the weight-gradient form: K long, split 8 ways, added into C32"""
    M, N, K = 1296, 256, 4096
    A, B, _ = _ops(M, N, K, 3)
    C = torch.ones((M, N), device="cuda")
    ib.gemm_bf16_nt(A, B, out32=C, accumulate=True, splits=8)
    ref = 1.0 + A.float() @ B.float().T
    assert float((C - ref).abs().max()) <= 1e-4 * float(ref.abs().max())


def test_gemm_strided_operands():
    """row strides larger than K (a view of a wider matrix)"""
    M, N, K = 200, 256, 136
    A, B, _ = _ops(M, N, 200, 4)
    A, B = A[:, :K], B[:, :K]
    C = torch.empty((M, N), device="cuda")
    ib.gemm_bf16_nt(A, B, out32=C)
    ref = A.float() @ B.float().T
    assert float((C - ref).abs().max()) <= 1e-4 * float(ref.abs().max())


def test_gemm_rejects_unaligned_k():
    A, B, _ = _ops(16, 16, 12, 5)
    C = torch.empty((16, 16), device="cuda")
    with pytest.raises(ib.IcxError) as ei:
        ib.gemm_bf16_nt(A, B, out32=C)
    assert ei.value.status == 1  # ICX_ERR_INVALID
