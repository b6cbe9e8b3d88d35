"""The GEMM tile-width autotuner: recorded widths are valid, every width gives the same output
bits, and a codec tuned on its first (eager) chunk codes the same bytes as an untuned one."""
import numpy as np
import pytest
import torch

from dcvc_b200 import _native as N, ops, synthetic
from tests.hts_fixtures import chunk, make_proxy, ref_frame, state_dict

pytestmark = pytest.mark.gpu

SHAPES = [  # (epilogue, M, N, K, sub_w, sub_cout)
    (N.EPI_BIAS, 8160, 512, 512, 0, 0),
    (N.EPI_BIAS_WSILU, 2040, 256, 512, 0, 0),
    (N.EPI_BIAS_RES, 4000, 512, 256, 0, 0),
    (N.EPI_QUAD, 2040, 1024, 512, 0, 0),
    (N.EPI_SUBPEL, 2040, 1024, 256, 60, 256),
]


@pytest.fixture(autouse=True)
def _clean_table():
    ops.gemm_tuning_clear()
    yield
    ops.gemm_autotune_enable(False)
    ops.gemm_tuning_clear()


@pytest.mark.parametrize("epi,M,Nn,K,sub_w,sub_cout", SHAPES)
def test_tuned_width_is_valid_and_bit_identical(epi, M, Nn, K, sub_w, sub_cout):
    assert ops.gemm_tuned(torch.float16, epi, M, Nn, K, sub_w) == 0
    bn, us = ops.gemm_autotune(torch.float16, epi, M, Nn, K, sub_w, sub_cout)
    torch.cuda.synchronize()
    assert bn in (256, 128, 64) and Nn % bn == 0 and us > 0
    if epi == N.EPI_QUAD:
        assert bn == 256
    assert ops.gemm_tuned(torch.float16, epi, M, Nn, K, sub_w) == bn
    g = torch.Generator(device="cuda").manual_seed(M + Nn + K)
    a = (torch.randn(M, K, device="cuda", generator=g) * 0.5).half()
    w = (torch.randn(Nn, K, device="cuda", generator=g) / K ** 0.5).half()
    b = None if epi == N.EPI_SUBPEL else torch.randn(Nn, device="cuda", generator=g) * 0.3
    res = torch.randn(M, Nn, device="cuda", generator=g).half() if epi == N.EPI_BIAS_RES else None
    kw = dict(sub_w=sub_w, sub_cout=sub_cout) if epi == N.EPI_SUBPEL else {}
    tuned = ops.conv1x1(a, w, b, epi, res, **kw)  # block_n = 0: the recorded width
    widths = [x for x in (256, 128, 64)
              if Nn % x == 0 and (epi != N.EPI_QUAD or x == 256)
              and (epi != N.EPI_SUBPEL or sub_cout % x == 0)]
    for x in widths:
        out = ops.conv1x1(a, w, b, epi, res, block_n=x, **kw)
        assert torch.equal(out.view(torch.int16), tuned.view(torch.int16)), x


def test_untunable_shape_and_clear():
    with pytest.raises(N.DcvcError):
        ops.gemm_autotune(torch.float16, N.EPI_BIAS, 1000, 200, 512)  # no width divides N
    ops.gemm_autotune(torch.float16, N.EPI_BIAS, 1000, 256, 512)
    assert ops.gemm_tuned(torch.float16, N.EPI_BIAS, 1000, 256, 512) != 0
    ops.gemm_tuning_clear()
    assert ops.gemm_tuned(torch.float16, N.EPI_BIAS, 1000, 256, 512) == 0


def test_codec_tunes_on_first_chunk_and_codes_the_same_bytes():
    H, W = 256, 256
    sd = state_dict()
    pr, pb = synthetic.padding_for(H, W)
    ref = ref_frame(H, W)
    xs = [chunk(H, W, 8 * k) for k in range(3)]

    def run():
        enc = make_proxy(sd)
        enc.add_ref_feature_from_frame(ref, True)
        out = [enc.compress(x, qp, False, pb, pr) for x, qp in zip(xs, (10, 40, 63))]
        torch.cuda.synchronize()
        return out

    plain = run()
    assert ops.gemm_tuned(torch.float16, N.EPI_QUAD, 1024, 1024, 512) == 0
    ops.gemm_autotune_enable(True)
    tuned = run()
    # the ffn.0 quad GEMM of a 512-channel block at H/8 x W/8 was tuned on the eager chunk
    assert ops.gemm_tuned(torch.float16, N.EPI_QUAD, 1024, 1024, 512) == 256
    for (b0, e0), (b1, e1) in zip(plain, tuned):
        assert e0 == e1 and np.array_equal(b0, b1)
