"""tcgen05 GEMM of the surrogate against a plain PyTorch FP32 reference.

The inputs are bf16, so the reference is the FP32 product of the same bf16
values; the tensor core accumulates in FP32, so the tolerance is FP32
summation-order rounding relative to the magnitude of the terms.
"""

import pytest
import torch

pytestmark = pytest.mark.gpu


def _ref(A, B):
    return A.float() @ B.float().t()


@pytest.mark.parametrize("M,N,K", [(128, 256, 64), (256, 256, 256), (200, 100, 48), (512, 16, 1024),
                                   (130, 512, 272), (1024, 256, 16)])
def test_gemm_matches_fp32_reference(M, N, K, cuda_device):
    from pyrite_b200 import mlp

    g = torch.Generator(device=cuda_device).manual_seed(M * 7 + N * 3 + K)
    A = torch.randn(M, K, device=cuda_device, generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, device=cuda_device, generator=g).to(torch.bfloat16)
    out = torch.full((M, N), float("nan"), device=cuda_device)
    status = torch.zeros(1, dtype=torch.int32, device=cuda_device)
    mlp.gemm(A, B, out_f32=out, status=status)
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    ref = _ref(A, B)
    scale = (A.float().abs() @ B.float().abs().t()).clamp_min(1.0)
    assert torch.all(torch.isfinite(out))
    assert float(((out - ref).abs() / scale).max()) < 1e-5


def test_gemm_epilogue_bias_silu_transposed(cuda_device):
    from pyrite_b200 import mlp

    M, N, K = 256, 256, 128
    g = torch.Generator(device=cuda_device).manual_seed(5)
    A = (0.2 * torch.randn(M, K, device=cuda_device, generator=g)).to(torch.bfloat16)
    B = (0.2 * torch.randn(N, K, device=cuda_device, generator=g)).to(torch.bfloat16)
    bias = torch.randn(N, device=cuda_device, generator=g)
    z = torch.empty(M, N, device=cuda_device)
    h = torch.empty(M, N, device=cuda_device, dtype=torch.bfloat16)
    ht = torch.empty(N, M, device=cuda_device, dtype=torch.bfloat16)
    mlp.gemm(A, B, bias=bias, act=1, out_f32=z, out_bf16=h, out_bf16_t=ht)
    zr = _ref(A, B) + bias
    hr = torch.nn.functional.silu(zr)
    torch.cuda.synchronize()
    assert float((z - zr).abs().max()) < 1e-3
    assert float((h.float() - hr).abs().max()) < 2e-2
    assert torch.equal(ht, h.t().contiguous())


def test_gemm_backward_epilogue(cuda_device):
    from pyrite_b200 import mlp

    M, N, K = 128, 256, 256
    g = torch.Generator(device=cuda_device).manual_seed(9)
    A = (0.1 * torch.randn(M, K, device=cuda_device, generator=g)).to(torch.bfloat16)
    B = (0.1 * torch.randn(N, K, device=cuda_device, generator=g)).to(torch.bfloat16)
    z = torch.randn(M, N, device=cuda_device, generator=g)
    out = torch.empty(M, N, device=cuda_device)
    mlp.gemm(A, B, dsilu_z=z, out_f32=out)
    t = torch.tanh(0.5 * z)
    ref = _ref(A, B) * (0.5 * (1 + t) + 0.25 * z * (1 - t * t))
    torch.cuda.synchronize()
    assert float((out - ref).abs().max()) < 3e-3 * float(ref.abs().max())
