"""tcgen05 tensor-core kernels of the learned preconditioner stage, checked
against FP32 matrix products of the same BF16-rounded operands."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _gemm(A, B):
    import torch

    from lowmachmixtures_b200 import _native
    lib = _native.load()
    M, K = A.shape
    N = B.shape[0]
    D = torch.empty(M, N, dtype=torch.float32, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = lib.lmm_nn_gemm_bf16(C.c_void_p(A.data_ptr()), C.c_void_p(B.data_ptr()), C.c_void_p(D.data_ptr()), M, N, K,
                              C.c_void_p(err.data_ptr()), C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 0
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    return D


@pytest.mark.parametrize("M,N,K", [(128, 16, 64), (300, 48, 200), (1000, 64, 432), (256, 256, 128), (64, 32, 8)])
def test_gemm_bf16_matches_fp32_product(M, N, K):
    import torch
    g = torch.Generator().manual_seed(M + N + K)
    A = torch.randn(M, K, generator=g).to(torch.bfloat16).cuda()
    B = torch.randn(N, K, generator=g).to(torch.bfloat16).cuda()
    D = _gemm(A, B)
    ref = A.float() @ B.float().t()
    np.testing.assert_allclose(D.cpu().numpy(), ref.cpu().numpy(), rtol=1e-4, atol=1e-3 * np.sqrt(K))
