"""The tensor-core BF16 GEMM (maf_bf16_gemm: tcgen05.mma, FP32 accumulation in
tensor memory) against an FP64 product of the same BF16 values, on shapes with
partial tiles in M, N and K."""
import ctypes as C

import pytest

M = pytest.importorskip("magnumaf")
torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("m,n,k", [(128, 32, 64), (300, 96, 200), (1000, 128, 1152), (77, 16, 8), (256, 200, 72),
                                   (4096, 64, 576)])
def test_bf16_gemm_matches_fp64_product(m, n, k):
    g = torch.Generator(device="cuda").manual_seed(m * 7 + n * 3 + k)
    A = torch.randn(m, k, device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn(n, k, device="cuda", generator=g).to(torch.bfloat16)
    out = torch.full((m, n), float("nan"), device="cuda", dtype=torch.float32)
    torch.cuda.synchronize()
    rc = M.lib.maf_bf16_gemm(C.c_void_p(A.data_ptr()), k, C.c_void_p(B.data_ptr()), k, C.c_void_p(out.data_ptr()),
                             n, m, n, k, None)
    assert rc == 0, M.lib.maf_last_error()
    torch.cuda.synchronize()
    ref = A.double() @ B.double().T
    # FP32 accumulation of k exact BF16 products
    err = ((out.double() - ref).abs().max() / ref.abs().max()).item()
    assert err < 5e-5, err


def test_bf16_gemm_rejects_unaligned_k():
    A = torch.zeros(16, 12, device="cuda", dtype=torch.bfloat16)
    out = torch.zeros(16, 16, device="cuda")
    rc = M.lib.maf_bf16_gemm(C.c_void_p(A.data_ptr()), 12, C.c_void_p(A.data_ptr()), 12, C.c_void_p(out.data_ptr()),
                             16, 16, 16, 12, None)
    assert rc == 1
