"""YUV 4:2:0 I/O on CPU: the oracle's conversions against the reference's own (golden fixtures
from tests/golden/make_yuv_golden.py), the reader / writer against the reference's file layout,
and the file-level helpers that need no GPU."""
import os
import sys

import numpy as np

from dcvc_b200 import synthetic
from dcvc_b200.video_io import YUV420Reader, YUV420Writer, frame_bytes, padding_size, write_yuv420

GOLD = os.path.join(os.path.dirname(__file__), "golden")
sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(__file__)), "oracle"))
import yuv_oracle  # noqa: E402


def test_oracle_matches_reference_conversions():
    g = np.load(os.path.join(GOLD, "yuv_golden.npz"))
    H, W, F, HP, WP = (int(v) for v in g["shape"])
    x = yuv_oracle.yuv420_to_input(g["planes"], F, H, W)
    assert np.array_equal(x.view(np.uint16), g["model_input"].view(np.uint16))
    rec = yuv_oracle.frames_to_yuv420(list(g["x_hat"]), H, W)
    assert np.array_equal(rec, g["rec_planes"])


def test_oracle_input_matches_synthetic_model_input():
    # the host path used by the tests and the bench (synthetic.to_model_input) is the same math
    frames = synthetic.video_chunk_yuv420(2, 32, 48, 3, 0)
    planes = np.concatenate([np.concatenate([y.ravel(), u.ravel(), v.ravel()]) for y, u, v in frames])
    x = yuv_oracle.yuv420_to_input(planes, 3, 32, 48)
    ref = synthetic.to_model_input(frames, device="cpu")[0].permute(1, 2, 0).numpy()
    assert np.array_equal(x.view(np.uint16), ref.view(np.uint16))


def test_reader_writer_round_trip(tmp_path):
    H, W = 24, 40
    frames = synthetic.video_chunk_yuv420(5, H, W, 5, 0)
    src = str(tmp_path / "in.yuv")
    assert write_yuv420(src, frames) == 5 * frame_bytes(W, H)
    with YUV420Reader(src, W, H, skip_frame=1) as r:
        y, uv = r.read_one_frame()
        assert y.shape == (1, H, W) and uv.shape == (2, H // 2, W // 2)
        assert np.array_equal(y[0], frames[1][0])
        assert np.array_equal(uv[0], frames[1][1]) and np.array_equal(uv[1], frames[1][2])
        raw = r.read_raw(8)  # only 3 frames left
        assert raw.size == 3 * frame_bytes(W, H) and r.eof
        assert r.read_one_frame() == (None, None)
    dst = str(tmp_path / "out.yuv")
    with YUV420Writer(dst, W, H) as w:
        w.write_one_frame(y, uv)
        w.write_raw(raw)
    with open(src, "rb") as a, open(dst, "rb") as b:
        assert a.read()[frame_bytes(W, H):] == b.read()


def test_padding_size_matches_reference_rule():
    assert padding_size(1080, 1920) == (0, 8)
    assert padding_size(240, 416) == (0, 0)
    assert padding_size(250, 410) == (6, 6)


def test_decode_sequence_rejects_an_undefined_sps(tmp_path):
    """A frame whose sps_id no earlier SPS unit defined is reported before any decoding (the
    reference's SPSHelper.get_sps_by_id returns None there and the harness fails on it)."""
    import pytest
    from dcvc_b200 import stream_helper as S
    from dcvc_b200.video_io import decode_sequence
    path = tmp_path / "bad.bin"
    with open(path, "wb") as f:
        S.write_sps(f, {"sps_id": 0, "height": 64, "width": 64})
        S.write_ip(f, True, 3, 20, 1, 0, b"\x00\x01\x02")
    with pytest.raises(ValueError, match="sps_id 3"):
        decode_sequence(str(path), 8, str(tmp_path / "rec.yuv"), None, None)
