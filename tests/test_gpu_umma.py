"""tcgen05 BF16 GEMM (shared-memory SW128 layout, descriptors, TMEM
epilogue) against a float32 torch product of the same bf16 inputs (gpu)."""
import numpy as np
import pytest
import torch

from ipc_warp_b200 import _native as N

pytestmark = pytest.mark.gpu


def umma_gemm(A, B):
    M, K = A.shape
    n = B.shape[0]
    C = torch.empty((M, n), dtype=torch.float32, device=A.device)
    st = torch.zeros(1, dtype=torch.int32, device=A.device)
    N.call("ipcb_umma_gemm_bf16", M, n, K, N.ptr(A), N.ptr(B), N.ptr(C), N.ptr(st), N.stream_handle())
    torch.cuda.synchronize()
    assert int(st.item()) == 0
    return C


@pytest.mark.parametrize("n,k", [(64, 64), (64, 192), (16, 64), (128, 128), (192, 64), (256, 256), (16, 256)])
@pytest.mark.parametrize("m", [1, 127, 128, 1000, 40_000])
def test_umma_gemm_matches_float32(cuda, m, n, k):
    g = torch.Generator(device=cuda).manual_seed(m * 7 + n + k)
    A = torch.randn((m, k), generator=g, device=cuda).to(torch.bfloat16)
    B = torch.randn((n, k), generator=g, device=cuda).to(torch.bfloat16)
    C = umma_gemm(A, B)
    ref = A.float() @ B.float().T
    err = (C - ref).abs().max().item()
    assert err <= 1e-4 * max(1.0, ref.abs().max().item()) * (k / 64), err


def test_umma_gemm_structured(cuda):
    """Identity and one-hot operands pin the row/column/K mapping exactly."""
    k = 128
    A = torch.zeros((256, k), device=cuda)
    A[torch.arange(256), torch.arange(256) % k] = 1.0
    B = torch.arange(64 * k, device=cuda, dtype=torch.float32).reshape(64, k) % 97
    C = umma_gemm(A.to(torch.bfloat16), B.to(torch.bfloat16))
    ref = (A @ B.T)
    assert torch.equal(C, ref)


def test_umma_gemm_rejects_unsupported_shapes(cuda):
    A = torch.zeros((4, 96), dtype=torch.bfloat16, device=cuda)
    B = torch.zeros((64, 96), dtype=torch.bfloat16, device=cuda)
    C = torch.zeros((4, 64), device=cuda)
    st = torch.zeros(1, dtype=torch.int32, device=cuda)
    rc = N.lib().ipcb_umma_gemm_bf16(4, 64, 96, N.ptr(A), N.ptr(B), N.ptr(C), N.ptr(st), N.stream_handle())
    assert rc == 1
