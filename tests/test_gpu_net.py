"""Kernels of the learned warm start: the tcgen05 GEMM (bf16 operands, fp32
accumulation in tensor memory) against a plain PyTorch fp32 matmul of the same
bf16 inputs."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _lib():
    from wavesim_b200 import _lib as L
    return L.lib


@pytest.mark.parametrize("M,N,K", [(128, 128, 64), (300, 200, 192), (1000, 32, 1728), (4096, 64, 896), (77, 130, 128)])
def test_gemm_bf16_matches_fp32_matmul(gpu, M, N, K):
    import torch
    lib = _lib()
    g = torch.Generator(device="cuda").manual_seed(M * 7 + N)
    A = torch.randn(M, K, device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, device="cuda", generator=g).to(torch.bfloat16)
    Cm = torch.zeros(M, N, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = lib.ws_gemm_bf16(A.data_ptr(), B.data_ptr(), Cm.data_ptr(), None, None, M, N, K, K, K, N, 0,
                          err.data_ptr(), None)
    torch.cuda.synchronize()
    assert rc == 0 and int(err.item()) == 0
    ref = A.float() @ B.float().t()
    assert float((Cm - ref).norm() / ref.norm()) < 1e-5


def test_gemm_bias_relu_epilogue(gpu):
    import torch
    lib = _lib()
    M, N, K = 256, 96, 128
    A = torch.randn(M, K, device="cuda").to(torch.bfloat16)
    B = torch.randn(N, K, device="cuda").to(torch.bfloat16)
    bias = torch.randn(N, device="cuda")
    out = torch.zeros(M, N, device="cuda", dtype=torch.bfloat16)
    rc = lib.ws_gemm_bf16(A.data_ptr(), B.data_ptr(), None, out.data_ptr(), bias.data_ptr(), M, N, K, K, K, N, 1,
                          None, None)
    torch.cuda.synchronize()
    assert rc == 0
    ref = torch.relu(A.float() @ B.float().t() + bias)
    assert float((out.float() - ref).norm() / ref.norm()) < 1e-2  # bf16 output rounding
