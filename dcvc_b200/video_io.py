"""YUV 4:2:0 file I/O and the end-to-end file round trip of the reference's test harness.

`YUV420Reader` / `YUV420Writer` have the interface of src/utils/video_reader.py:51-99 and
src/utils/video_writer.py:33-61 (planar I420, 8-bit: Y then U then V per frame).  Their
`read_raw` / `write_raw` methods move whole frames as bytes, which is what the device path uses:
the 8-bit planes cross PCIe and `ops.yuv420_to_input` / `ops.frames_to_yuv420` do the
conversions of get_src_frame (test_video.py:69-123) and of the decoded-frame writer
(test_video.py:355-362) on the GPU.

`encode_sequence` / `decode_sequence` follow run_one_point_with_stream (test_video.py:167-405):
an intra frame first (and every `intra_period` frames), then P calls of `frames_per_call` frames
(8 for the HT-S / HT-L chunk codecs, 1 for the LD codec) with the reference's reset schedule; the
bitstream is the reference's NAL container (SPS, then one I or P unit per call,
dcvc_b200.stream_helper).
"""
import io
import os

import numpy as np
import torch

from . import ops
from .stream_helper import (NalType, SPSHelper, read_header, read_ip_remaining,
                            read_sps_remaining, write_ip, write_sps)


def frame_bytes(width, height):
    return width * height * 3 // 2


class _I420File:
    """Frame geometry of a planar 8-bit I420 file: frame k occupies bytes
    [k * frame, (k + 1) * frame), luma plane first, then the two chroma planes."""

    def __init__(self, width, height):
        self.width, self.height = width, height
        self.luma = width * height
        self.frame = frame_bytes(width, height)

    def split(self, buf):
        """One frame's bytes -> (y [1, H, W], uv [2, H/2, W/2]) views of a private array."""
        a = np.frombuffer(buf, dtype=np.uint8).copy()
        y = a[: self.luma].reshape(1, self.height, self.width)
        uv = a[self.luma: self.frame].reshape(2, self.height // 2, self.width // 2)
        return y, uv


class YUV420Reader:
    """Reads frames of a planar 8-bit YUV 4:2:0 file by position.

    The constructor and `read_one_frame` keep the interface of the reference's reader
    (src/utils/video_reader.py:50-99): a path without the ".yuv" suffix gets it appended,
    `skip_frame` frames are passed over, and `read_one_frame` returns (y [1, H, W],
    uv [2, H/2, W/2]) or (None, None) once the file has no whole frame left.  Internally the
    reader keeps only a frame cursor and reads each request with one positioned read
    (`os.pread`) of whole frames, so `read_raw` can hand many frames to the device path in one
    buffer."""

    def __init__(self, src_path, width, height, skip_frame=0):
        self.src_path = src_path if src_path.endswith(".yuv") else src_path + ".yuv"
        self.geom = _I420File(width, height)
        self._fd = os.open(self.src_path, os.O_RDONLY)
        self._frames_in_file = os.fstat(self._fd).st_size // self.geom.frame
        self.cursor = max(0, int(skip_frame))
        self.eof = self.cursor >= self._frames_in_file

    def _take(self, n):
        k = max(0, min(n, self._frames_in_file - self.cursor))
        data = os.pread(self._fd, k * self.geom.frame, self.cursor * self.geom.frame) if k else b""
        self.cursor += k
        self.eof = k < n
        return data, k

    def read_one_frame(self):
        """(y [1, H, W], uv [2, H/2, W/2]) uint8 arrays, or (None, None) at the end."""
        if self.eof:
            return None, None
        data, k = self._take(1)
        if k == 0:
            return None, None
        return self.geom.split(data)

    def read_raw(self, n):
        """Up to n whole frames as one uint8 array (frames back to back); fewer at the end."""
        if self.eof:
            return np.zeros(0, dtype=np.uint8)
        data, _ = self._take(n)
        return np.frombuffer(data, dtype=np.uint8).copy()

    def __enter__(self):
        return self

    def __exit__(self, exc_type, exc_val, exc_tb):
        self.close()
        return False

    def __del__(self):
        self.close()

    def close(self):
        fd = getattr(self, "_fd", None)
        if fd is not None:
            os.close(fd)
            self._fd = None


class YUV420Writer:
    """Appends planar 8-bit YUV 4:2:0 frames to a file.

    Path rule of the reference's writer (src/utils/video_writer.py:33-61): a destination that
    does not end in ".yuv" names a directory, and the frames go to "out.yuv" inside it.  Frames
    are accumulated as byte chunks and appended with one `os.write` per call."""

    def __init__(self, dst_path, width, height):
        self.dst_path = dst_path if dst_path.endswith(".yuv") else os.path.join(dst_path, "out.yuv")
        self.geom = _I420File(width, height)
        self._fd = os.open(self.dst_path, os.O_WRONLY | os.O_CREAT | os.O_TRUNC, 0o644)

    def _append(self, *arrays):
        payload = b"".join(np.ascontiguousarray(a, dtype=np.uint8).tobytes() for a in arrays)
        view = memoryview(payload)
        while view:
            view = view[os.write(self._fd, view):]

    def write_one_frame(self, y, uv):
        if np.size(y) + np.size(uv) != self.geom.frame:
            raise ValueError(f"frame of {np.size(y) + np.size(uv)} bytes, expected "
                             f"{self.geom.frame} for {self.geom.width}x{self.geom.height}")
        self._append(y, uv)

    def write_raw(self, planes):
        """Whole I420 frames back to back (a uint8 array or tensor)."""
        if isinstance(planes, torch.Tensor):
            planes = planes.cpu().numpy()
        if np.size(planes) % self.geom.frame:
            raise ValueError("write_raw takes whole frames")
        self._append(planes)

    def __enter__(self):
        return self

    def __exit__(self, exc_type, exc_val, exc_tb):
        self.close()
        return False

    def __del__(self):
        self.close()

    def close(self):
        fd = getattr(self, "_fd", None)
        if fd is not None:
            os.close(fd)
            self._fd = None


def padding_size(height, width, p=16):
    """(padding_r, padding_b) as DMCI.get_padding_size (common_model.py:103-108)."""
    return (width + p - 1) // p * p - width, (height + p - 1) // p * p - height


def _is_intra(frame_idx, intra_period):
    # test_video.py:207-213
    intra = frame_idx == 0 or intra_period == 1
    if intra_period > 1 and frame_idx != 1 and frame_idx % intra_period == 1:
        intra = True
    return intra


def _upload(raw, device):
    host = torch.from_numpy(raw).pin_memory()
    return host.to(device, non_blocking=True)


def encode_sequence(src_path, width, height, frame_num, bin_path, i_proxy, p_proxy, qp_i, qp_p,
                    frames_per_call=8, intra_period=-1, reset_interval=32, device="cuda"):
    """Codes `frame_num` frames of a YUV 4:2:0 file into the NAL bitstream `bin_path`.

    i_proxy: a DMCIProxy; p_proxy: a DMCHTSProxy / DMCHTLProxy (frames_per_call 8) or DMCLDProxy
    (frames_per_call 1), both with parameters set.  Returns per-call records
    (frame index, kind, frames, bytes)."""
    pad_r, pad_b = padding_size(height, width)
    fb = frame_bytes(width, height)
    out = io.BytesIO()
    sps_helper = SPSHelper()
    records = []
    with YUV420Reader(src_path, width, height) as reader:
        frame_idx = 0
        while frame_idx < frame_num:
            intra = _is_intra(frame_idx, intra_period)
            n = 1 if intra else min(frames_per_call, frame_num - frame_idx)
            raw = reader.read_raw(n)
            if raw.size != n * fb:
                raise EOFError(f"{src_path}: fewer than {frame_num} frames")
            calls = 1 if intra else frames_per_call
            if calls > n:  # the last chunk repeats its last frame (test_video.py:101-107)
                raw = np.concatenate([raw] + [raw[(n - 1) * fb:]] * (calls - n))
            x = ops.yuv420_to_input(_upload(raw, device), calls, height, width)
            if intra:
                qp, reset = qp_i, 0
                bits, x_hat, ecp = i_proxy.compress(x, qp, pad_b, pad_r)
                p_proxy.add_ref_feature_from_frame(x_hat, True)
            else:
                reset = 1 if reset_interval > 0 and \
                    (frame_idx + frames_per_call) % reset_interval == 1 else 0
                qp = qp_p
                bits, ecp = p_proxy.compress(x, qp, bool(reset), pad_b, pad_r)
            sps = {"sps_id": -1, "height": height, "width": width}
            sps_id, sps_new = sps_helper.get_sps_id(sps)
            sps["sps_id"] = sps_id
            nb = write_sps(out, sps) if sps_new else 0
            nb += write_ip(out, intra, sps_id, qp, ecp, reset, bits)
            records.append((frame_idx, "I" if intra else "P", n, nb))
            frame_idx += n
    with open(bin_path, "wb") as f:
        f.write(out.getbuffer())
    return records


def decode_sequence(bin_path, frame_num, rec_path, i_proxy, p_proxy, frames_per_call=8):
    """Decodes a bitstream written by encode_sequence and writes the reconstruction as a YUV
    4:2:0 file (the decoded-frame writer of test_video.py:355-362).  Returns the number of
    frames written."""
    with open(bin_path, "rb") as f:
        buf = io.BytesIO(f.read())
    sps_helper = SPSHelper()
    writer = None
    decoded = 0
    try:
        while decoded < frame_num:
            header = read_header(buf)
            while header["nal_type"] == NalType.NAL_SPS:
                sps_helper.add_sps_by_id(read_sps_remaining(buf, header["sps_id"]))
                header = read_header(buf)
            sps = sps_helper.get_sps_by_id(header["sps_id"])
            if sps is None:
                raise ValueError(f"frame {decoded} references sps_id {header['sps_id']}, which no "
                                 "preceding SPS unit defines")
            H, W = sps["height"], sps["width"]
            if writer is None:
                writer = YUV420Writer(rec_path, W, H)
            qp, ec_part, reset, bits = read_ip_remaining(buf)
            bits = np.frombuffer(bits, dtype=np.uint8)
            if header["nal_type"] == NalType.NAL_I:
                x_hat = i_proxy.decompress(bits, qp, H, W, ec_part)
                p_proxy.add_ref_feature_from_frame(x_hat, False)
                frames, n = [x_hat], 1
            else:
                out = p_proxy.decompress(bits, qp, H, W, ec_part, bool(reset))
                frames = out if isinstance(out, list) else [out]
                n = min(frames_per_call, frame_num - decoded)
            writer.write_raw(ops.frames_to_yuv420(frames[:n], H, W))
            decoded += n
    finally:
        if writer is not None:
            writer.close()
    return decoded


def write_yuv420(path, frames):
    """Writes uint8 (y, u, v) plane triples (synthetic.video_chunk_yuv420's frames) to a file."""
    with open(path, "wb") as f:
        for y, u, v in frames:
            f.write(np.ascontiguousarray(y, dtype=np.uint8).tobytes())
            f.write(np.ascontiguousarray(u, dtype=np.uint8).tobytes())
            f.write(np.ascontiguousarray(v, dtype=np.uint8).tobytes())
    return os.path.getsize(path)
