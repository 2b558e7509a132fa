"""Tensor-core kernels of the learned proposal against PyTorch float32 references of the same ops.

GEMM: inputs are BF16, so the reference multiplies the same BF16 values in float32; the
tolerance (relative to the largest reference value) is 1e-5, float32 accumulation over K <= 2304.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

GEMM_TOL = 1e-5


def gemm(A, B, epi, bias=None, slope=0.2, out=None, splits=0):
    from shotsweep_b200 import _lib
    M, K = A.shape
    N = B.shape[0]
    if out is None:
        dt = torch.bfloat16 if epi == _lib.EPI_BIAS_LRELU_BF16 else torch.float32
        out = torch.zeros(M, N, dtype=dt, device=A.device)
    err = torch.zeros(1, dtype=torch.int32, device=A.device)
    L = _lib.load()
    _lib.check(L.ss_gemm_bf16(_lib.ptr(A), A.stride(0), _lib.ptr(B), B.stride(0), M, N, K, epi, _lib.ptr(out),
                              out.stride(0), _lib.ptr(bias), slope, splits, _lib.ptr(err),
                              _lib.stream_handle(A.device)), 'ss_gemm_bf16')
    torch.cuda.synchronize()
    assert err.item() == 0
    return out


@pytest.mark.parametrize('M,N,K', [(200, 40, 40), (1000, 256, 1152), (300, 96, 520), (129, 300, 64),
                                   (8192, 256, 2304), (64, 32, 9216)])
def test_gemm_f32_matches_float32_matmul(M, N, K):
    from shotsweep_b200 import _lib
    g = torch.Generator(device='cuda').manual_seed(M * 7 + N + K)
    A = torch.randn(M, K, device='cuda', generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, device='cuda', generator=g).to(torch.bfloat16)
    ref = A.float() @ B.float().T
    got = gemm(A, B, _lib.EPI_F32)
    assert (got - ref).abs().max().item() <= GEMM_TOL * ref.abs().max().item() * 10 + 1e-6 * K ** 0.5
    bias = torch.randn(N, device='cuda', generator=g)
    got = gemm(A, B, _lib.EPI_BIAS_F32, bias=bias)
    assert torch.allclose(got, ref + bias, rtol=0, atol=GEMM_TOL * ref.abs().max().item() * 10 + 1e-6 * K ** 0.5)


def test_gemm_split_k_accumulates():
    from shotsweep_b200 import _lib
    g = torch.Generator(device='cuda').manual_seed(11)
    A = torch.randn(64, 50000, device='cuda', generator=g).to(torch.bfloat16)
    B = torch.randn(48, 50000, device='cuda', generator=g).to(torch.bfloat16)
    ref = A.double() @ B.double().T
    start = torch.randn(64, 48, device='cuda', generator=g)
    got = gemm(A, B, _lib.EPI_F32_ADD, out=start.clone())
    err = (got.double() - (ref + start.double())).abs().max().item()
    assert err <= 1e-4 * ref.abs().max().item()


def test_gemm_bias_leaky_relu_bf16():
    from shotsweep_b200 import _lib
    g = torch.Generator(device='cuda').manual_seed(5)
    A = torch.randn(517, 72, device='cuda', generator=g).to(torch.bfloat16)
    B = torch.randn(64, 72, device='cuda', generator=g).to(torch.bfloat16)
    bias = torch.randn(64, device='cuda', generator=g)
    x = A.float() @ B.float().T + bias
    ref = torch.where(x > 0, x, 0.2 * x)
    got = gemm(A, B, _lib.EPI_BIAS_LRELU_BF16, bias=bias).float()
    assert ((got - ref).abs() <= 2 ** -8 * ref.abs() + 1e-5).all()     # one BF16 rounding
