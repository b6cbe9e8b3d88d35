"""GPU YUV 4:2:0 I/O: the conversion kernels bit-exact against the reference's conversions (golden
fixtures), the oracle, and the reference harness's torch expressions run on the device; and the
end-to-end file round trip (YUV file -> NAL bitstream -> YUV file) through the intra and HT-S
proxies."""
import os
import sys

import numpy as np
import pytest
import torch

from dcvc_b200 import ops, synthetic
from dcvc_b200.video_io import decode_sequence, encode_sequence, frame_bytes, write_yuv420
from tests.hts_fixtures import make_proxy, state_dict
from tests.intra_fixtures import intra_state_dict, make_intra_proxy

GOLD = os.path.join(os.path.dirname(__file__), "golden")
sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(__file__)), "oracle"))
import yuv_oracle  # noqa: E402

pytestmark = pytest.mark.gpu


def _hwc(x):
    return x[0].permute(1, 2, 0).cpu().numpy()


def test_kernels_match_reference_golden():
    g = np.load(os.path.join(GOLD, "yuv_golden.npz"))
    H, W, F, HP, WP = (int(v) for v in g["shape"])
    x = ops.yuv420_to_input(torch.from_numpy(g["planes"]).cuda(), F, H, W)
    assert np.array_equal(_hwc(x).view(np.uint16), g["model_input"].view(np.uint16))
    frames = [torch.from_numpy(f).cuda().permute(2, 0, 1)[None] for f in g["x_hat"]]
    rec = ops.frames_to_yuv420(frames, H, W).cpu().numpy()
    assert np.array_equal(rec, g["rec_planes"])


@pytest.mark.parametrize("H,W,F", [(1080, 1920, 8), (250, 410, 1), (64, 96, 3)])
def test_kernels_match_oracle_and_torch(H, W, F):
    rng = np.random.default_rng(H + W + F)
    planes = rng.integers(0, 256, F * frame_bytes(W, H)).astype(np.uint8)
    x = ops.yuv420_to_input(torch.from_numpy(planes).cuda(), F, H, W)
    assert x.shape == (1, 3 * F, H, W)
    assert np.array_equal(_hwc(x).view(np.uint16),
                          yuv_oracle.yuv420_to_input(planes, F, H, W).view(np.uint16))
    # the reference harness's expressions on the device (test_video.py:355-362)
    Hp, Wp = (H + 15) // 16 * 16, (W + 15) // 16 * 16
    g = torch.Generator(device="cuda").manual_seed(3)
    frames = [((torch.rand(1, Hp, Wp, 3, device="cuda", generator=g) - 0.5) * 1.02).half()
              .clamp(-0.5, 0.5).permute(0, 3, 1, 2) for _ in range(F)]
    rec = ops.frames_to_yuv420(frames, H, W).cpu().numpy()
    ref = []
    for f in frames:
        xh = f[:, :, :H, :W] + 0.5
        y = torch.clamp(xh[:, :1] * 255, 0, 255).round().byte()
        uv = torch.clamp(torch.nn.functional.avg_pool2d(xh[:, 1:], 2, 2) * 255, 0, 255).byte()
        ref += [y.reshape(-1).cpu().numpy(), uv.reshape(-1).cpu().numpy()]
    assert np.array_equal(rec, np.concatenate(ref))
    orc = yuv_oracle.frames_to_yuv420([f[0].permute(1, 2, 0).cpu().numpy() for f in frames], H, W)
    assert np.array_equal(rec, orc)


def test_bad_arguments_raise():
    from dcvc_b200._native import DcvcError
    p = torch.zeros(frame_bytes(10, 10), dtype=torch.uint8, device="cuda")
    with pytest.raises(DcvcError):
        ops.yuv420_to_input(p, 9, 10, 10)  # more than 8 frames
    with pytest.raises(DcvcError):
        ops.yuv420_to_input(p, 1, 9, 10)  # odd height


def test_file_round_trip(tmp_path):
    H, W, N = 72, 112, 11  # I frame, one 8-frame chunk, one 2-frame chunk (padded to 8)
    frames = synthetic.video_chunk_yuv420(2, H, W, N, 0)
    src, binp, rec = (str(tmp_path / n) for n in ("src.yuv", "s.bin", "rec.yuv"))
    write_yuv420(src, frames)
    i_enc, i_dec = make_intra_proxy(intra_state_dict()), make_intra_proxy(intra_state_dict())
    p_enc, p_dec = make_proxy(state_dict()), make_proxy(state_dict())
    # reset_interval 8: the first P chunk resets the temporal memory
    recs = encode_sequence(src, W, H, N, binp, i_enc, p_enc, 30, 30, reset_interval=8)
    assert [r[1] for r in recs] == ["I", "P", "P"] and [r[2] for r in recs] == [1, 8, 2]
    assert os.path.getsize(binp) == sum(r[3] for r in recs)
    assert decode_sequence(binp, N, rec, i_dec, p_dec) == N
    assert os.path.getsize(rec) == N * frame_bytes(W, H)
    # the decoded file equals the decoder's reconstructions converted on the host by the oracle
    i2, p2 = make_intra_proxy(intra_state_dict()), make_proxy(state_dict())
    from dcvc_b200.stream_helper import read_header, read_ip_remaining, read_sps_remaining
    import io
    buf = io.BytesIO(open(binp, "rb").read())
    out = []
    for k in range(3):
        h = read_header(buf)
        if h["nal_type"] == 0:
            read_sps_remaining(buf, h["sps_id"])
            h = read_header(buf)
        qp, ecp, reset, bits = read_ip_remaining(buf)
        bits = np.frombuffer(bits, dtype=np.uint8)
        if k == 0:
            xh = i2.decompress(bits, qp, H, W, ecp)
            p2.add_ref_feature_from_frame(xh, False)
            fr = [xh]
        else:
            fr = p2.decompress(bits, qp, H, W, ecp, bool(reset))[: recs[k][2]]
        out.append(yuv_oracle.frames_to_yuv420([f[0].permute(1, 2, 0).cpu().numpy() for f in fr], H, W))
    assert open(rec, "rb").read() == np.concatenate(out).tobytes()
