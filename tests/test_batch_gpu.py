"""Packed batches of the HT-S codec: n streams of one resolution coded by one handle, every
network layer one launch over the n stacked images.  Each stream's payload bytes, latents and
reconstructions must be bitwise those of a single-stream codec on the same inputs and QPs: the
stacked depthwise convolutions keep each image's own zero border, the checkerboard masks each
image's own row parity (odd latent heights included), the x q epilogues each stream's own QP
rows, the hyper path each image's own replicate padding, and the compaction each stream's own
symbols."""
import numpy as np
import pytest
import torch

from dcvc_b200 import synthetic
from tests.hts_fixtures import state_dict

pytestmark = pytest.mark.gpu


def _proxy(sd, precision):
    from dcvc_b200.inference_extensions_cuda import DMCHTSProxy
    p = DMCHTSProxy(precision)
    p.set_param(sd, 0.15)
    return p


@pytest.mark.parametrize("H,W,n,precision", [(240, 416, 3, "fp16"), (200, 248, 2, "bf16"),
                                             (128, 192, 4, "fp8")])
def test_packed_batch_equals_single_streams(H, W, n, precision):
    sd = state_dict()
    pr, pb = synthetic.padding_for(H, W)
    seeds = [2 + k for k in range(n)]
    refs = [synthetic.padded_reference_frame(synthetic.video_chunk_yuv420(s, H, W, 1, 0)[0])
            for s in seeds]
    qp_plan = [[(5 + 23 * k) % 64 for k in range(n)], [(40 + 11 * k) % 64 for k in range(n)]]
    chunks = [[synthetic.to_model_input(synthetic.video_chunk_yuv420(s, H, W, 8, 8 * c))
               for s in seeds] for c in range(2)]
    # one stream at a time
    single = []
    for k in range(n):
        enc, dec = _proxy(sd, precision), _proxy(sd, precision)
        enc.add_ref_feature_from_frame(refs[k], True)
        dec.add_ref_feature_from_frame(refs[k], False)
        res = []
        for c in range(2):
            bits, ecp = enc.compress(chunks[c][k], qp_plan[c][k], False, pb, pr)
            frames = dec.decompress(bits, qp_plan[c][k], H, W, ecp, False)
            torch.cuda.synchronize()
            res.append((bits, ecp, [f.clone() for f in frames], enc.buffer("y_q").clone()))
        single.append(res)
    # all n streams in one packed batch
    enc, dec = _proxy(sd, precision), _proxy(sd, precision)
    enc.add_ref_features_from_frames(refs, True)
    dec.add_ref_features_from_frames(refs, False)
    for c in range(2):
        out = enc.compress_batch(chunks[c], qp_plan[c], False, pb, pr)
        frames = dec.decompress_batch([b for b, _ in out], qp_plan[c], H, W, [e for _, e in out],
                                      False)
        torch.cuda.synchronize()
        y_q = enc.buffer("y_q")
        rows = y_q.shape[0] // n
        for k in range(n):
            bits, ecp, sframes, sy = single[k][c]
            assert out[k][1] == ecp and np.array_equal(out[k][0], bits), (c, k)
            assert torch.equal(y_q[k * rows:(k + 1) * rows].view(torch.int16), sy.view(torch.int16))
            for i in range(8):
                assert torch.equal(frames[i][k:k + 1], sframes[i]), (c, k, i)
        for name in ("common", "y_q", "y_hat", "feature_p"):
            assert torch.equal(enc.buffer(name).view(torch.int16), dec.buffer(name).view(torch.int16))


def test_batch_arguments_are_checked():
    from dcvc_b200._native import DcvcError
    sd = state_dict()
    H, W = 64, 64
    enc = _proxy(sd, "fp16")
    refs = [synthetic.padded_reference_frame(synthetic.video_chunk_yuv420(2, H, W, 1, 0)[0])] * 2
    enc.add_ref_features_from_frames(refs, True)
    x = synthetic.to_model_input(synthetic.video_chunk_yuv420(2, H, W, 8, 0))
    with pytest.raises(DcvcError):
        enc.compress_batch([x, x, x], [1, 2, 3], False, 0, 0)  # 3 inputs for 2 streams
    with pytest.raises(DcvcError):
        enc.compress_batch([x, x], [1, 64], False, 0, 0)  # qp out of range
    out = enc.compress_batch([x, x], [7, 7], False, 0, 0)
    assert np.array_equal(out[0][0], out[1][0])  # same input, same QP, same reference: same bytes


def test_packed_batch_with_and_without_depthwise_fusion():
    """Stacked images keep their own zero borders in the depthwise form of the residual GEMM
    too: a packed batch codes to the same bytes with the depthwise 3x3 fused or separate."""
    from dcvc_b200 import _native as N
    sd = state_dict()
    H, W, n = 200, 248, 2
    pr, pb = synthetic.padding_for(H, W)
    refs = [synthetic.padded_reference_frame(synthetic.video_chunk_yuv420(4 + k, H, W, 1, 0)[0])
            for k in range(n)]
    xs = [synthetic.to_model_input(synthetic.video_chunk_yuv420(4 + k, H, W, 8, 8)) for k in range(n)]
    out = {}
    try:
        for on in (1, 0):
            N.lib.dcvc_dw_fusion(on)
            enc = _proxy(sd, "fp16")
            enc.add_ref_features_from_frames(refs, True)
            out[on] = enc.compress_batch(xs, [7, 58], False, pb, pr)
            torch.cuda.synchronize()
    finally:
        N.lib.dcvc_dw_fusion(0)
    for (b0, e0), (b1, e1) in zip(out[0], out[1]):
        assert e0 == e1 and np.array_equal(b0, b1)
