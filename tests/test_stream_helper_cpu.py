"""The NAL container (dcvc_b200/stream_helper.py) against bytes written by the reference's
stream_helper (tests/golden/nal_golden.json), and its reader on those bytes."""
import hashlib
import io
import json
import os
import sys

import pytest

from dcvc_b200 import stream_helper as S

GOLD = os.path.join(os.path.dirname(__file__), "golden", "nal_golden.json")
sys.path.insert(0, os.path.dirname(GOLD))
from make_nal_golden import payload  # noqa: E402


def _write_all(gold):
    f = io.BytesIO()
    helper = S.SPSHelper()
    sizes = []
    for i, u in enumerate(gold["sequence"]):
        if u[0] == "sps":
            sps = {"sps_id": -1, "height": u[1], "width": u[2]}
            sid, new = helper.get_sps_id(sps)
            sps["sps_id"] = sid
            sizes.append(["sps", sid, new, S.write_sps(f, sps) if new else 0])
        else:
            _, is_i, sid, qp, ec, reset, n = u
            sizes.append(["ip", S.write_ip(f, is_i, sid, qp, ec, reset, payload(i, n))])
    return f.getvalue(), sizes


@pytest.fixture(scope="module")
def gold():
    return json.load(open(GOLD))


def test_writer_matches_reference_bytes(gold):
    data, sizes = _write_all(gold)
    assert sizes == gold["written"]
    assert len(data) == gold["size"] and data[:64].hex() == gold["head"]
    assert hashlib.sha256(data).hexdigest() == gold["sha256"]


def test_reader_parses_reference_bytes(gold):
    data, _ = _write_all(gold)
    f = io.BytesIO(data)
    helper = S.SPSHelper()
    want = [[u[1], u[2], u[3], u[4], u[5], payload(i, u[6])] for i, u in enumerate(gold["sequence"])
            if u[0] == "ip"]
    got = []
    while f.tell() < len(data):
        h = S.read_header(f)
        if h["nal_type"] == S.NalType.NAL_SPS:
            helper.add_sps_by_id(S.read_sps_remaining(f, h["sps_id"]))
            continue
        qp, ec, reset, body = S.read_ip_remaining(f)
        got.append([h["nal_type"] == S.NalType.NAL_I, h["sps_id"], qp, ec, reset, body])
    assert got == want
    assert helper.get_sps_by_id(1) == {"sps_id": 1, "height": 720, "width": 1280}


def test_truncated_unit_raises():
    f = io.BytesIO()
    S.write_ip(f, False, 0, 10, 3, 0, b"\x01" * 300)
    data = f.getvalue()[:-5]
    r = io.BytesIO(data)
    S.read_header(r)
    with pytest.raises(EOFError):
        S.read_ip_remaining(r)


def test_varint_edges():
    for v in (0, 127, 128, 16383, 16384, (1 << 30) - 1):
        f = io.BytesIO()
        S.write_uint_adaptive(f, v)
        f.seek(0)
        assert S.read_uint_adaptive(f) == v
    with pytest.raises(ValueError):
        S.write_uint_adaptive(io.BytesIO(), 1 << 30)
