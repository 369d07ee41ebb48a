"""The warm-start network's tensor-core kernels against an FP32 reference of
the same operation (torch on the same bf16 inputs)."""
from __future__ import annotations

import pytest

torch = pytest.importorskip("torch")

from bowshock_b200 import _native  # noqa: E402

pytestmark = pytest.mark.gpu


def _gemm(a, b, c, splits=1, accumulate=False):
    lib = _native.load()
    m, k = a.shape
    n = b.shape[0]
    _native.check(lib.bs_gemm_bf16(a.data_ptr(), b.data_ptr(), c.data_ptr(), m, n, k, splits,
                                   1 if accumulate else 0, torch.cuda.current_stream().cuda_stream), lib)


@pytest.mark.parametrize("m,n,k", [(128, 64, 64), (256, 256, 128), (200, 128, 256), (384, 256, 512),
                                   (1000, 256, 256)])
def test_gemm_matches_fp32_reference(m, n, k):
    g = torch.Generator(device="cuda").manual_seed(m * 7 + n * 3 + k)
    a = torch.randn(m, k, device="cuda", generator=g).to(torch.bfloat16)
    b = torch.randn(n, k, device="cuda", generator=g).to(torch.bfloat16)
    c = torch.full((m, n), float("nan"), device="cuda")
    _gemm(a, b, c)
    ref = a.double() @ b.double().T
    err = (c.double() - ref).abs().max().item()
    # Exact bf16 products, FP32 sums in a different order: ~1e-6 of sqrt(k).
    assert err <= 1e-4 * k ** 0.5, err


def test_split_k_accumulates():
    g = torch.Generator(device="cuda").manual_seed(5)
    m, n, k = 256, 256, 1024
    a = torch.randn(m, k, device="cuda", generator=g).to(torch.bfloat16)
    b = torch.randn(n, k, device="cuda", generator=g).to(torch.bfloat16)
    c = torch.ones(m, n, device="cuda")
    _gemm(a, b, c, splits=4, accumulate=True)
    ref = 1.0 + a.double() @ b.double().T
    assert (c.double() - ref).abs().max().item() <= 1e-4 * k ** 0.5
