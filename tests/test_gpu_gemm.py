"""spx_gemm_bf16 (tcgen05.mma, TMEM accumulators) against an fp32 matmul of the same bf16 operands.

Shapes cover the warm-start MLP's forward (batch x 1024 -> 256, 256 -> 256, 256 -> 7) and
weight-gradient GEMMs (reduction over the batch), ragged M, N and K, and every epilogue option.
Tolerance: f32 accumulation of bf16 products in a different order than torch's, so a few f32 ulps
of the row-sum magnitude.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _gemm(a, b, *, scale=1.0, bias=None, relu=False, mask=None, out_f32=True, out_bf16=False, out_t=False,
          accumulate_into=None):
    import torch

    from imageprocessor_new_b200 import _lib

    m, k = a.shape
    n = b.shape[0]
    outs = {}
    ep = _lib.GemmEpilogue()
    ep.scale = scale
    if bias is not None:
        ep.bias = bias.data_ptr()
    ep.relu = int(relu)
    if mask is not None:
        ep.mask_act, ep.ld_mask = mask.data_ptr(), mask.shape[1]
    if out_f32:
        outs["f32"] = accumulate_into if accumulate_into is not None else torch.full((m, n), np.nan,
                                                                                     device="cuda")
        ep.out_f32, ep.ld_f32, ep.accumulate = outs["f32"].data_ptr(), n, int(accumulate_into is not None)
    if out_bf16:
        outs["bf16"] = torch.empty((m, n), dtype=torch.bfloat16, device="cuda")
        ep.out_bf16, ep.ld_bf16 = outs["bf16"].data_ptr(), n
    if out_t:
        outs["t"] = torch.empty((n, m), dtype=torch.bfloat16, device="cuda")
        ep.out_bf16_t, ep.ld_t = outs["t"].data_ptr(), m
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    _lib.call("spx_gemm_bf16", a.data_ptr(), a.stride(0), b.data_ptr(), b.stride(0), m, n, k, ep, err.data_ptr(),
              torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    return outs


@pytest.mark.parametrize("m,n,k", [(128, 256, 64), (300, 256, 1024), (4096, 256, 256), (256, 256, 4096),
                                   (4096, 7, 256), (77, 300, 200), (1, 16, 8), (640, 48, 1000)])
def test_gemm_matches_fp32_matmul(m, n, k):
    import torch

    g = torch.Generator(device="cuda").manual_seed(m * 7 + n * 13 + k)
    a = torch.randn((m, k), device="cuda", generator=g).to(torch.bfloat16)
    b = torch.randn((n, k), device="cuda", generator=g).to(torch.bfloat16)
    want = a.float() @ b.float().T
    got = _gemm(a, b)["f32"]
    scale = (a.float().abs() @ b.float().abs().T) * 2.0 ** -20 + 1e-6
    assert torch.all((got - want).abs() <= scale), float(((got - want).abs() / scale).max())


def test_gemm_epilogues():
    import torch

    g = torch.Generator(device="cuda").manual_seed(5)
    m, n, k = 333, 256, 320
    a = torch.randn((m, k), device="cuda", generator=g).to(torch.bfloat16)
    b = torch.randn((n, k), device="cuda", generator=g).to(torch.bfloat16)
    bias = torch.randn(n, device="cuda", generator=g)
    mask = torch.randn((m, n), device="cuda", generator=g).to(torch.bfloat16)
    base = (a.float() @ b.float().T) * 0.5 + bias
    tol = (a.float().abs() @ b.float().abs().T) * 2.0 ** -20 + 1e-5
    o = _gemm(a, b, scale=0.5, bias=bias, relu=True, out_bf16=True, out_t=True)
    want = torch.relu(base)
    assert torch.all((o["f32"] - want).abs() <= tol)
    assert torch.equal(o["bf16"], o["f32"].to(torch.bfloat16))
    assert torch.equal(o["t"], o["bf16"].T.contiguous())
    o = _gemm(a, b, scale=0.5, bias=bias, mask=mask)
    want = torch.where(mask.float() > 0, base, torch.zeros_like(base))
    assert torch.all((o["f32"] - want).abs() <= tol)
    acc = torch.ones((m, n), device="cuda")
    o = _gemm(a, b, accumulate_into=acc)
    assert torch.all((o["f32"] - (1.0 + a.float() @ b.float().T)).abs() <= tol + 1e-6)


def test_gemm_rejects_bad_strides():
    import torch

    from imageprocessor_new_b200 import _lib

    a = torch.zeros((8, 12), dtype=torch.bfloat16, device="cuda")
    ep = _lib.GemmEpilogue()
    out = torch.zeros((8, 8), device="cuda")
    ep.out_f32, ep.ld_f32, ep.scale = out.data_ptr(), 8, 1.0
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    with pytest.raises(_lib.LibraryError):
        _lib.call("spx_gemm_bf16", a.data_ptr(), 12, a.data_ptr(), 12, 8, 8, 12, ep, err.data_ptr(), 0)
