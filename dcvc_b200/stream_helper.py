"""NAL-style container around the rANS payloads, byte-compatible with the reference's
src/utils/stream_helper.py (write_sps :144-154, write_ip :130-141, read_header :37-56,
read_sps_remaining :83-88, read_ip_remaining :74-81, adaptive-length integers :59-127,
NalType :157-160, SPSHelper :163-192).

Layout of one unit:
  SPS: [nal_type(4) | sps_id(4)] [height varint] [width varint]
  I/P: [nal_type(4) | sps_id(4)] [qp] [ec_part(7) | reset_feature_memory(1)] [len varint] [payload]
varint: < 2^7 in 1 byte (top bit 0); < 2^14 in 2 bytes (top bits 10); < 2^30 in 4 bytes (top bits 11),
big-endian.
"""
import enum
import struct


class NalType(enum.IntEnum):
    NAL_SPS = 0
    NAL_I = 1
    NAL_P = 2


def _put(f, data):
    f.write(bytes(data))
    return len(data)


def _get(f, n):
    b = f.read(n)
    if len(b) != n:
        raise EOFError("truncated bitstream")
    return b


def write_uint_adaptive(f, a):
    if a < 0:
        raise ValueError("negative value")
    if a < (1 << 7):
        return _put(f, [a])
    if a < (1 << 14):
        return _put(f, [0x80 | (a >> 8), a & 0xff])
    if a >= (1 << 30):
        raise ValueError("value too large for the adaptive integer format")
    return _put(f, [0xC0 | (a >> 24), (a >> 16) & 0xff, (a >> 8) & 0xff, a & 0xff])


def read_uint_adaptive(f):
    b0 = _get(f, 1)[0]
    if b0 >> 7 == 0:
        return b0
    b1 = _get(f, 1)[0]
    if b0 >> 6 == 0x02:
        return ((b0 & 0x3F) << 8) | b1
    b2, b3 = _get(f, 2)
    return ((b0 & 0x3F) << 24) | (b1 << 16) | (b2 << 8) | b3


def write_sps(f, sps):
    if not 0 <= sps["sps_id"] < 16:
        raise ValueError("sps_id must be in [0, 16)")
    n = _put(f, [(int(NalType.NAL_SPS) << 4) | sps["sps_id"]])
    n += write_uint_adaptive(f, sps["height"])
    n += write_uint_adaptive(f, sps["width"])
    return n


def write_ip(f, is_i_frame, sps_id, qp, ec_part, reset_feature_memory, bit_stream):
    if not 0 <= qp < 256:
        raise ValueError("qp must fit one byte")
    nal = NalType.NAL_I if is_i_frame else NalType.NAL_P
    n = _put(f, [(int(nal) << 4) + sps_id, qp, (ec_part << 1) + reset_feature_memory])
    n += write_uint_adaptive(f, len(bit_stream))
    f.write(bytes(bit_stream))
    return n + len(bit_stream)


def read_header(f):
    flag = _get(f, 1)[0]
    nal_type = flag >> 4
    header = {"nal_type": NalType(nal_type)} if nal_type < 3 else {"nal_type": nal_type}
    if nal_type < 3:
        header["sps_id"] = flag & 0x0F
        return header
    frame_num = (flag & 0x0F) + 1
    ids = []
    for _ in range(0, frame_num, 2):
        b = _get(f, 1)[0]
        ids += [b >> 4, b & 0x0F]
    header["frame_num"] = frame_num
    header["sps_ids"] = ids[:frame_num]
    return header


def read_sps_remaining(f, sps_id):
    return {"sps_id": sps_id, "height": read_uint_adaptive(f), "width": read_uint_adaptive(f)}


def read_ip_remaining(f):
    qp, flag = struct.unpack(">BB", _get(f, 2))
    length = read_uint_adaptive(f)
    return qp, (flag >> 1) & 0x7F, flag & 0x01, _get(f, length)


class SPSHelper:
    """Assigns sps ids to picture sizes (first unused id for a new size, at most 16)."""

    def __init__(self):
        self.spss = []

    def add_sps_by_id(self, sps):
        for i, s in enumerate(self.spss):
            if s["sps_id"] == sps["sps_id"]:
                self.spss[i] = dict(sps)
                return
        self.spss.append(dict(sps))

    def get_sps_by_id(self, sps_id):
        for s in self.spss:
            if s["sps_id"] == sps_id:
                return s
        return None

    def get_sps_id(self, target):
        top = -1
        for s in self.spss:
            if s["height"] == target["height"] and s["width"] == target["width"]:
                return s["sps_id"], False
            top = max(top, s["sps_id"])
        if top >= 15:
            raise ValueError("more than 16 picture sizes in one stream")
        sps = dict(target)
        sps["sps_id"] = top + 1
        self.spss.append(sps)
        return sps["sps_id"], True
