"""rANS coder parity on CPU: the product coder (libdcvc_b200.so) and the C oracle against the
reference coder's golden bytes (tests/golden/rans_golden.npz, made by make_golden.py from the
reference sources), plus round trips, edge cases and corrupt-stream handling."""
import ctypes
import os

import numpy as np
import pytest

from dcvc_b200 import MLCodec_extensions_cpp as M
from tests.oracle_loader import oracle_lib

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


@pytest.fixture(scope="module")
def gold():
    g = np.load(os.path.join(GOLD, "rans_golden.npz"))
    qps = g["qz_qps"].tolist()
    # rebuild a full-size z table array: the fixture keeps only the QPs its cases use
    qz = np.zeros((64 * 128, g["qz"].shape[1]), np.int32)
    lz = np.full(64 * 128, 3, np.int32)
    qz[:, 1] = 65535
    qz[:, 2] = 65536
    for j, q in enumerate(qps):
        qz[q * 128:(q + 1) * 128] = g["qz"][j * 128:(j + 1) * 128]
        lz[q * 128:(q + 1) * 128] = g["lz"][j * 128:(j + 1) * 128]
    cases = []
    for i in range(int(g["ncases"])):
        ny, nz, ecp, qp = g[f"c{i}_meta"].tolist()
        cases.append((ny, nz, ecp, qp, g[f"c{i}_y"], g[f"c{i}_z"], g[f"c{i}_bytes"]))
    return g["qy"], g["ly"], qz, lz, cases


def _coders(qy, ly, qz, lz):
    enc, dec = M.RansEncoder(), M.RansDecoder()
    for c in (enc, dec):
        c.set_cdf(qz, lz, 0)
        c.set_cdf(qy, ly, 1)
    return enc, dec


def test_product_matches_reference_bytes(gold):
    qy, ly, qz, lz, cases = gold
    enc, dec = _coders(qy, ly, qz, lz)
    for ny, nz, ecp, qp, y, z, ref in cases:
        enc.set_entropy_coder_parallel(ecp)
        enc.reset()
        enc.encode_y(y)
        enc.encode_z(z, qp * 128, 128)
        enc.flush()
        out = enc.get_encoded_stream()
        assert out.dtype == np.uint8 and out.tobytes() == ref.tobytes(), (ny, nz, ecp)
        dec.set_entropy_coder_parallel(ecp)
        dec.set_stream(ref)
        dec.decode_z(nz, qp * 128, 128)
        assert (dec.get_decoded_tensor() == z).all()
        dec.decode_y((y & 0xff).astype(np.uint8))
        assert (dec.get_decoded_tensor() == (y >> 8).astype(np.int8)).all()


def test_oracle_matches_reference_bytes(gold):
    qy, ly, qz, lz, cases = gold
    lib = oracle_lib()
    for ny, nz, ecp, qp, y, z, ref in cases:
        cap = (ny + nz) * 4 + 1024
        buf = np.zeros(cap, np.uint8)
        n = lib.oracle_encode(_p(qz), _p(lz), qz.shape[1], _p(qy), _p(ly), qy.shape[1], _p(y), ny,
                              _p(z), nz, qp * 128, 128, ecp, _p(buf), cap)
        assert n == ref.size and buf[:n].tobytes() == ref.tobytes(), (ny, nz, ecp)
        yo = np.zeros(max(ny, 1), np.int8)
        zo = np.zeros(max(nz, 1), np.int8)
        idx = (y & 0xff).astype(np.uint8)
        rc = lib.oracle_decode(_p(qz), _p(lz), qz.shape[1], _p(qy), _p(ly), qy.shape[1], _p(ref),
                               ref.size, _p(idx), ny, nz, qp * 128, 128, ecp, _p(yo), _p(zo))
        assert rc == 0
        assert (yo[:ny] == (y >> 8).astype(np.int8)).all() and (zo[:nz] == z).all()


def test_multi_segment_order(gold):
    """Several y segments then z (the intra model's order); decode in reverse order."""
    qy, ly, qz, lz, _ = gold
    enc, dec = _coders(qy, ly, qz, lz)
    rng = np.random.default_rng(5)
    segs = []
    for n in (3000, 1, 0, 4096):
        idx = rng.integers(0, 128, n)
        val = np.clip(np.round(rng.standard_normal(n) * 3), -128, 127).astype(np.int64)
        segs.append(((val << 8) + idx).astype(np.int16))
    z = rng.integers(-64, 64, 510).astype(np.int8)
    for ecp in (1, 3, 8):
        enc.set_entropy_coder_parallel(ecp)
        enc.reset()
        for s in segs:
            enc.encode_y(s)
        enc.encode_z(z, 128 * 7, 128)
        enc.flush()
        data = enc.get_encoded_stream()
        dec.set_entropy_coder_parallel(ecp)
        dec.set_stream(data)
        dec.decode_z(z.size, 128 * 7, 128)
        assert (dec.get_decoded_tensor() == z).all()
        for s in reversed(segs):
            dec.decode_y((s & 0xff).astype(np.uint8))
            assert (dec.get_decoded_tensor() == (s >> 8).astype(np.int8)).all()


def test_truncated_stream_is_an_error(gold):
    qy, ly, qz, lz, cases = gold
    enc, dec = _coders(qy, ly, qz, lz)
    ny, nz, ecp, qp, y, z, ref = cases[0]
    dec.set_entropy_coder_parallel(ecp)
    dec.set_stream(ref[: ref.size // 3])
    with pytest.raises(RuntimeError):
        dec.decode_z(nz, qp * 128, 128)
        dec.decode_y((y & 0xff).astype(np.uint8))


def test_bad_header_is_an_error(gold):
    qy, ly, qz, lz, cases = gold
    _, dec = _coders(qy, ly, qz, lz)
    bad = np.zeros(16, np.uint8)
    bad[:4] = np.frombuffer(np.int32(1 << 20).tobytes(), np.uint8)  # offset past the payload
    dec.set_entropy_coder_parallel(3)
    with pytest.raises(RuntimeError):
        dec.set_stream(bad)


def test_bad_parallelism_rejected(gold):
    enc = M.RansEncoder()
    with pytest.raises(ValueError):
        enc.set_entropy_coder_parallel(9)


def test_ec_parallel_rule():
    assert [M.ec_parallel_for(n) for n in (0, 32767, 32768, 65536 * 3, 10 ** 7)] == [1, 1, 1, 6, 8]


def test_pmf_to_quantized_cdf_matches_reference():
    g = np.load(os.path.join(GOLD, "pmf_golden.npz"))
    lib = oracle_lib()
    for i in range(int(g["n"])):
        p, ref = g[f"p{i}"], g[f"c{i}"]
        assert M.pmf_to_quantized_cdf(p) == ref.tolist()
        out = np.zeros(p.size + 1, np.uint32)
        assert lib.oracle_pmf_to_quantized_cdf(_p(p), p.size, _p(out)) == p.size + 1
        assert (out == ref).all()


@pytest.mark.parametrize("sub_stream", [0, 3])
def test_worker_exception_is_reported_and_the_coder_recovers(gold, sub_stream):
    """A fault injected into one sub-stream task (as a failed allocation in a worker would
    throw) fails the call with DCVC_INTERNAL instead of terminating the process; the other tasks
    finish, and the next call on the same coder produces the reference bytes again.  Task 0 runs
    on the calling thread, task 3 on a worker."""
    from dcvc_b200 import _native as N
    qy, ly, qz, lz, cases = gold
    ny, nz, ecp, qp, y, z, ref = max(cases, key=lambda c: c[2])  # the most sub-streams
    assert ecp > sub_stream
    enc, dec = _coders(qy, ly, qz, lz)
    enc.set_entropy_coder_parallel(ecp)
    dec.set_entropy_coder_parallel(ecp)

    def encode():
        enc.reset()
        enc.encode_y(y)
        enc.encode_z(z, qp * 128, 128)
        enc.flush()
        return enc.get_encoded_stream()

    M.inject_task_fault(sub_stream)
    with pytest.raises(N.DcvcError, match="injected fault") as ei:
        encode()
    assert ei.value.status == 8  # DCVC_INTERNAL
    assert encode().tobytes() == ref.tobytes()

    dec.set_stream(ref)
    M.inject_task_fault(sub_stream)
    with pytest.raises(N.DcvcError, match="injected fault") as ei:
        dec.decode_z(nz, qp * 128, 128)
    assert ei.value.status == 8  # DCVC_INTERNAL
    dec.set_stream(ref)
    dec.decode_z(nz, qp * 128, 128)
    assert np.array_equal(dec.get_decoded_tensor(), z)
    M.inject_task_fault(-1)


def test_long_bypass_runs_in_corrupt_payloads_decode_like_the_oracle():
    """Random payloads decoded under a table whose escape symbol covers all but one code point:
    nearly every symbol takes the 2-bit bypass path, so runs of 16 digits (which can set bit 31
    of the escaped value, making it negative) occur.  The product decoder and the C oracle must
    give the same symbols for every one of them, including the negative-value cases."""
    lib = oracle_lib()
    qz = np.zeros((1, 3), np.int32)
    qz[0] = [0, 1, 65536]
    lz = np.array([3], np.int32)
    qy, ly = qz.copy(), lz.copy()
    enc, dec = _coders(qy, ly, qz, lz)
    rng = np.random.default_rng(11)
    n = 40000
    negative_cases = 0
    for trial in range(6):
        data = rng.integers(0, 256, 1 << 20).astype(np.uint8)
        dec.set_entropy_coder_parallel(1)
        dec.set_stream(data)
        dec.decode_z(n, 0, 1)
        got = dec.get_decoded_tensor().copy()
        zo = np.zeros(n, np.int8)
        yo = np.zeros(1, np.int8)
        idx = np.zeros(1, np.uint8)
        rc = lib.oracle_decode(_p(qz), _p(lz), qz.shape[1], _p(qy), _p(ly), qy.shape[1],
                               _p(data), data.size, _p(idx), 0, n, 0, 1, 1, _p(yo), _p(zo))
        assert rc == 0
        assert np.array_equal(got, zo), trial
        negative_cases += int((np.abs(got.astype(np.int32)) > 64).sum())
    assert negative_cases > 0  # long runs were exercised, not only short escapes
