"""The chunk server on the GPU: every result is the same alone and in the mix.

Streams of three sizes, encoders and a decoder, run first one at a time (one stream in the
server) and then all at once with their requests interleaved across slots.  The kernels are
deterministic (no atomics, no split-K) and each stream's temporal context lives in its own
session, so the payload bytes and the decoded I420 planes must be identical, byte for byte."""
import numpy as np
import pytest
import torch

from tests.hts_fixtures import SKIP_THRES, ref_frame, state_dict
from dcvc_b200 import synthetic
from dcvc_b200.serving import ChunkServer, HtsSessionFactory, StreamSpec, pack_i420

pytestmark = pytest.mark.gpu

SIZES = [(128, 192), (200, 248), (96, 160)]
QPS = [7, 50, 33]  # three chunks: the third starts a new group (gop 2) and re-seeds


def _factory(sd, refs):
    return HtsSessionFactory(sd, SKIP_THRES, refs, gop=2, copy_output=True)


def _server(f, slots, budget=150e9):
    return ChunkServer(f.open, f.estimate_bytes, slots=slots, hbm_budget=budget,
                       on_worker_start=f.worker_start)


def _content(H, W):
    return [pack_i420(synthetic.video_chunk_yuv420(2, H, W, 8, 8 * k)) for k in range(2)]


def test_results_are_the_same_alone_and_in_the_mix():
    sd = state_dict()
    refs = {s: ref_frame(*s) for s in SIZES}
    content = {s: _content(*s) for s in SIZES}
    torch.cuda.synchronize()

    # alone: one encoder stream per size, then a decoder of the first size's payloads
    alone_bytes = {}
    for s in SIZES:
        srv = _server(_factory(sd, refs), slots=1)
        srv.open_stream(s, StreamSpec("enc", *s))
        reqs = [srv.submit(s, qp, content[s][k % 2]) for k, qp in enumerate(QPS)]
        alone_bytes[s] = [r.wait(300) for r in reqs]
        srv.shutdown()
    dec_size = SIZES[0]
    srv = _server(_factory(sd, refs), slots=1)
    srv.open_stream("dec", StreamSpec("dec", *dec_size))
    reqs = [srv.submit("dec", qp, alone_bytes[dec_size][k]) for k, qp in enumerate(QPS)]
    alone_planes = [r.wait(300) for r in reqs]
    srv.shutdown()
    H, W = dec_size
    for p in alone_planes:
        assert p.dtype == np.uint8 and p.size == 8 * H * W * 3 // 2
    assert not np.array_equal(alone_planes[0], alone_planes[1])

    # in the mix: all streams at once, requests interleaved, four slots
    f = _factory(sd, refs)
    srv = _server(f, slots=4)
    for s in SIZES:
        srv.open_stream(s, StreamSpec("enc", *s))
    srv.open_stream("dec", StreamSpec("dec", *dec_size))
    mix = {s: [] for s in SIZES}
    mix_dec = []
    for k, qp in enumerate(QPS):
        for s in SIZES:
            mix[s].append(srv.submit(s, qp, content[s][k % 2]))
        mix_dec.append(srv.submit("dec", qp, alone_bytes[dec_size][k]))
    for s in SIZES:
        for k, r in enumerate(mix[s]):
            bits, ecp = r.wait(300)
            a_bits, a_ecp = alone_bytes[s][k]
            assert ecp == a_ecp and np.array_equal(bits, a_bits), (s, k)
    for k, r in enumerate(mix_dec):
        assert np.array_equal(r.wait(300), alone_planes[k]), k
    assert srv.max_sessions == 4
    assert srv.failed == 0 and srv.completed == 4 * len(QPS)
    held = srv.held_bytes()
    assert held > 0
    srv.shutdown()
    assert srv.held_bytes() == 0
    # the measured session sizes now drive the admission estimates
    assert f.estimate_bytes(StreamSpec("enc", *SIZES[0])) > 0


def test_admission_by_budget_on_the_gpu():
    """A budget that fits one session: the second stream starts only after the first closes,
    and both results are still exact."""
    sd = state_dict()
    s = SIZES[2]
    refs = {s: ref_frame(*s)}
    content = _content(*s)
    f = _factory(sd, refs)
    srv = _server(f, slots=2)
    srv.open_stream("probe", StreamSpec("enc", *s))
    probe = srv.submit("probe", 20, content[0]).wait(300)
    srv.shutdown()
    one = f.estimate_bytes(StreamSpec("enc", *s))
    srv = _server(f, slots=2, budget=int(one * 1.5))
    srv.open_stream("a", StreamSpec("enc", *s))
    srv.open_stream("b", StreamSpec("enc", *s))
    ra = srv.submit("a", 20, content[0])
    rb = srv.submit("b", 20, content[0])
    bits_a, _ = ra.wait(300)
    assert srv.sessions() == 1 and not rb.finished()
    srv.close_stream("a")
    bits_b, _ = rb.wait(300)
    srv.shutdown()
    assert np.array_equal(bits_a, probe[0]) and np.array_equal(bits_b, probe[0])
    assert srv.peak_held <= srv.hbm_budget
