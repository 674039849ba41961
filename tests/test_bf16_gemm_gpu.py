"""The tcgen05 BF16 GEMM (D = A B^T, FP32 accumulation in tensor memory)
against an FP64 product of the same BF16 inputs.  BF16 x BF16 products are
exact in FP32, so the only error is FP32 summation: |D - D64| <= k * eps32 *
sum_k |a||b|."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("m,n,k", [(128, 64, 64), (256, 128, 128), (384, 64, 192), (128, 128, 512)])
def test_bf16_gemm_matches_fp64(native, ctx, m, n, k):
    import torch
    g = torch.Generator().manual_seed(m * 7 + n + k)
    a = torch.randn(m, k, generator=g).to(torch.bfloat16)
    b = torch.randn(n, k, generator=g).to(torch.bfloat16)
    da, db = a.cuda(), b.cuda()
    dd = torch.full((m, n), float("nan"), device="cuda")
    torch.cuda.synchronize()
    native.bf16_gemm_nt(ctx, da.data_ptr(), db.data_ptr(), dd.data_ptr(), m, n, k)
    got = dd.cpu().double().numpy()
    a64, b64 = a.double().numpy(), b.double().numpy()
    ref = a64 @ b64.T
    bound = k * np.finfo(np.float32).eps * (np.abs(a64) @ np.abs(b64).T) + 1e-30
    assert np.isfinite(got).all()
    assert (np.abs(got - ref) <= bound).all(), np.abs(got - ref).max()


def test_bf16_gemm_rejects_bad_shapes(native, ctx):
    import torch
    a = torch.zeros(128, 64, dtype=torch.bfloat16, device="cuda")
    d = torch.zeros(128, 64, device="cuda")
    for m, n, k in [(100, 64, 64), (128, 32, 64), (128, 64, 48)]:
        with pytest.raises(native.OwtkError):
            native.bf16_gemm_nt(ctx, a.data_ptr(), a.data_ptr(), d.data_ptr(), m, n, k)
