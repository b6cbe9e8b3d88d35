"""Fused ConvFFN kernel (dcvc_conv_ffn): bit-identical with the two GEMMs it replaces (the quad
GEMM, then the residual GEMM, each through dcvc_conv1x1) over block widths, quad widths, ragged
pixel counts, output pitches and the x q epilogue; unsupported shapes are rejected."""
import pytest
import torch

from dcvc_b200 import _native as N
from dcvc_b200 import ops

pytestmark = pytest.mark.gpu


def _weights(C, cffn, g):
    w1 = (torch.randn(4 * cffn, C, device="cuda", generator=g) * C ** -0.5).half()
    b1 = torch.randn(4 * cffn, device="cuda", generator=g) * 0.1
    w2 = (torch.randn(C, cffn, device="cuda", generator=g) * cffn ** -0.5).half()
    b2 = torch.randn(C, device="cuda", generator=g) * 0.1
    return w1, b1, w2, b2


@pytest.mark.parametrize("bn", [0, 128, 256])
@pytest.mark.parametrize("M,C,cffn,with_q,pitch", [
    (32640, 512, 256, False, 0), (1000, 512, 256, True, 0), (8160, 256, 128, False, 0),
    (777, 256, 128, True, 0), (4096, 768, 256, False, 0), (2000, 256, 128, False, 512)])
def test_fused_matches_two_gemms(M, C, cffn, with_q, pitch, bn):
    g = torch.Generator(device="cuda").manual_seed(M + C + cffn)
    x = torch.randn(M, C, device="cuda", generator=g).half()
    w1, b1, w2, b2 = _weights(C, cffn, g)
    if cffn == 256 and bn == 256:
        # two 64 KB q buffers leave room for 128-wide items only
        with pytest.raises(N.DcvcError):
            ops.conv_ffn(x, w1, b1, w2, b2, block_n=bn)
        return
    q = (torch.rand(C, device="cuda", generator=g) + 0.5).half() if with_q else None
    quad = ops.conv1x1(x, w1, b1, N.EPI_QUAD)
    epi = N.EPI_BIAS_RES_Q if with_q else N.EPI_BIAS_RES
    ref = ops.conv1x1(quad, w2, b2, epi, res=x, qscale=q)
    if pitch:
        buf = torch.full((M, pitch), float("nan"), device="cuda", dtype=torch.float16)
        out = ops.conv_ffn(x, w1, b1, w2, b2, qscale=q, out=buf[:, 64:64 + C], block_n=bn)
        assert torch.isnan(buf[:, :64]).all() and torch.isnan(buf[:, 64 + C:]).all()
    else:
        out = ops.conv_ffn(x, w1, b1, w2, b2, qscale=q, block_n=bn)
    torch.cuda.synchronize()
    assert N.device_error() == 0
    assert torch.equal(out.view(torch.int16), ref.view(torch.int16))


def test_fused_twice_in_a_row_and_in_place_inputs_untouched():
    g = torch.Generator(device="cuda").manual_seed(7)
    x = torch.randn(3000, 512, device="cuda", generator=g).half()
    x0 = x.clone()
    w = _weights(512, 256, g)
    a = ops.conv_ffn(x, *w)
    b = ops.conv_ffn(x, *w)
    assert torch.equal(a, b) and torch.equal(x, x0)


def test_unsupported_shapes_rejected():
    g = torch.Generator(device="cuda").manual_seed(1)
    x = torch.randn(256, 384, device="cuda", generator=g).half()
    w = _weights(384, 192, g)
    with pytest.raises(N.DcvcError):
        ops.conv_ffn(x, *w)
