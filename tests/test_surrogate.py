"""The tensor-core (tcgen05) BF16 GEMM of the sky-bin visibility surrogate
against torch's FP32 product of the same bf16 inputs."""
import pytest


@pytest.mark.gpu
@pytest.mark.parametrize("M,N,K", [(128, 128, 64), (256, 384, 320), (384, 256, 1024)])
def test_gemm_bf16_matches_fp32_product(M, N, K):
    import torch
    from solargpu_b200 import api
    g = torch.Generator(device="cuda").manual_seed(M + N + K)
    A = torch.randn(M, K, device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, device="cuda", generator=g).to(torch.bfloat16)
    bias = torch.randn(N, device="cuda", generator=g)
    want = A.float() @ B.float().T
    got = api.gemm_bf16(A, B)
    torch.cuda.synchronize()
    torch.testing.assert_close(got, want, rtol=1e-4, atol=1e-3)
    got2 = api.gemm_bf16(A, B, bias=bias, relu=True)
    torch.testing.assert_close(got2, torch.relu(want + bias), rtol=1e-4, atol=1e-3)
    hb = torch.empty(M, N, dtype=torch.bfloat16, device="cuda")
    api.gemm_bf16(A, B, out_bf16=hb, bias=bias)
    torch.testing.assert_close(hb.float(), (want + bias).to(torch.bfloat16).float(), rtol=1e-2, atol=1e-2)


def test_gemm_rejects_bad_shapes():
    from solargpu_b200 import api
    import ctypes as C
    rc = api.lib().solar_gpu_gemm_bf16(C.c_void_p(16), C.c_void_p(32), C.c_void_p(64), None, None, 100, 128, 64, 0,
                                       None)
    assert rc in (-1, -2, -3)
