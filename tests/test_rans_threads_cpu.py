"""Host rANS coder under concurrency: the coder keeps persistent worker threads per calling thread,
so several streams coding at once (one host thread each, as the batched serving form runs them)
and a process forked after the coder has run must all produce the reference's bytes."""
import os
import threading

import numpy as np
import pytest

from dcvc_b200 import MLCodec_extensions_cpp as M
from dcvc_b200.entropy_tables import gaussian_tables


def _tables():
    qy, ly = gaussian_tables()
    return qy, ly, np.tile(qy[:1], (128, 1)).astype(np.int32), np.tile(ly[:1], 128).astype(np.int32)


_TABLES = _tables()  # built once: a forked child must not run torch (its thread pool is not fork-safe)


def _payload(seed, ecp):
    qy, ly, qz, lz = _TABLES
    rng = np.random.default_rng(seed)
    q = np.clip(np.round(rng.laplace(0, 2.0, 150000)), -128, 127).astype(np.int64)
    y = ((q << 8) + rng.integers(0, 128, q.size)).astype(np.int16)
    z = np.clip(np.round(rng.laplace(0, 1.5, 128 * 60)), -64, 63).astype(np.int8)
    enc = M.RansEncoder()
    enc.set_cdf(qz, lz, 0)
    enc.set_cdf(qy, ly, 1)
    enc.set_entropy_coder_parallel(ecp)
    enc.encode_y(y)
    enc.encode_z(z, 0, 128)
    enc.flush()
    out = enc.get_encoded_stream().tobytes()
    dec = M.RansDecoder()
    dec.set_cdf(qz, lz, 0)
    dec.set_cdf(qy, ly, 1)
    dec.set_entropy_coder_parallel(ecp)
    dec.set_stream(np.frombuffer(out, dtype=np.uint8))
    dec.decode_z(z.size, 0, 128)
    assert np.array_equal(dec.get_decoded_tensor(), z)
    dec.decode_y((y & 0xff).astype(np.uint8))
    assert np.array_equal(dec.get_decoded_tensor(), (y >> 8).astype(np.int8))
    return out


def test_concurrent_callers_match_serial():
    ref = {(s, e): _payload(s, e) for s in range(3) for e in (1, 3, 8)}
    got, errors = {}, []

    def run(seed, ecp):
        try:
            for _ in range(3):
                got[(seed, ecp)] = _payload(seed, ecp)
        except Exception as exc:  # pragma: no cover - reported below
            errors.append(exc)

    threads = [threading.Thread(target=run, args=k) for k in ref]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors
    assert got == ref


@pytest.mark.filterwarnings("ignore::DeprecationWarning")  # fork() with the coder's threads alive
def test_forked_child_codes_the_same_bytes():
    ref = _payload(5, 8)  # the parent's worker threads now exist
    r, w = os.pipe()
    pid = os.fork()
    if pid == 0:  # child: its own pool, same bytes
        try:
            ok = _payload(5, 8) == ref
        except Exception:
            ok = False
        os.write(w, b"1" if ok else b"0")
        os._exit(0)
    os.close(w)
    res = os.read(r, 1)
    os.close(r)
    os.waitpid(pid, 0)
    assert res == b"1"
