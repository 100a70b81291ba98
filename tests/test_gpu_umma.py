"""The tcgen05 tensor-core GEMM (BF16 x BF16 -> FP32 in TMEM) against a plain
PyTorch FP32 matmul of the same BF16 operands."""
import ctypes as C

import pytest

pytestmark = pytest.mark.gpu


def _gemm(lib, A, B, M, N, K, grid_x, splits):
    import torch
    out = torch.empty((splits, M, N) if splits > 1 else (M, N), dtype=torch.float32, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    lib.cl_umma_gemm_bf16.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int,
                                      C.c_int, C.c_int, C.c_void_p, C.c_void_p]
    lib.cl_umma_gemm_bf16.restype = C.c_int
    rc = lib.cl_umma_gemm_bf16(A.data_ptr(), B.data_ptr(), out.data_ptr(), M, N, K, grid_x, splits,
                               err.data_ptr(), None)
    torch.cuda.synchronize()
    assert rc == 0
    assert int(err.item()) == 0, "tensor-core completion wait ran out"
    return out.sum(0) if splits > 1 else out


@pytest.mark.parametrize("M,N,K,grid_x,splits", [
    (128, 32, 64, 1, 1),
    (256, 256, 256, 2, 1),
    (512, 192, 128, 3, 1),
    (1024, 256, 256, 4, 1),
    (256, 256, 1024, 2, 4),
    (2048, 256, 256, 3, 1),      # 16 tiles over 3 CTAs: both accumulators reused
    (2560, 192, 192, 2, 1),
])
def test_umma_gemm_matches_torch(M, N, K, grid_x, splits):
    import torch
    from crysplight_b200 import _lib
    lib = _lib.load()
    g = torch.Generator(device="cuda").manual_seed(M + N + K)
    A = torch.randn(M, K, device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, device="cuda", generator=g).to(torch.bfloat16)
    ref = A.float() @ B.float().T
    got = _gemm(lib, A, B, M, N, K, grid_x, splits)
    err = (got - ref).abs().max().item()
    scale = ref.abs().max().item()
    print(M, N, K, "max abs err", err, "scale", scale)
    assert err <= 1e-4 * scale + 1e-3
