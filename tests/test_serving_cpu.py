"""Chunk server scheduling on the CPU with fake sessions: per-stream order, concurrency bounded by
the slots, admission by the device-memory budget, error delivery and shutdown."""
import threading
import time

import numpy as np
import pytest

from dcvc_b200.serving import ChunkServer, StreamSpec, latency_summary, poisson_arrivals


class FakeFactory:
    """Sessions whose run() sleeps `work` seconds and records what ran where."""

    def __init__(self, work=0.01, bytes_per_px=1.0, fail_open=(), fail_run=()):
        self.work = work
        self.bytes_per_px = bytes_per_px
        self.fail_open = set(fail_open)
        self.fail_run = set(fail_run)
        self.lock = threading.Lock()
        self.running = set()        # stream ids with a request in flight
        self.max_concurrent = 0
        self.overlap_same_stream = False
        self.log = []               # (stream_id, seq) in completion order
        self.opened = []
        self.closed = []
        self.live = 0
        self.max_live_bytes = 0
        self.live_bytes = 0

    def estimate(self, spec):
        return int(spec.height * spec.width * self.bytes_per_px)

    def open(self, sid, spec):
        if sid in self.fail_open:
            raise RuntimeError(f"cannot open {sid}")
        f = self

        class S:
            device_bytes = f.estimate(spec)

            def run(self, req):
                with f.lock:
                    if req.stream_id in f.running:
                        f.overlap_same_stream = True
                    f.running.add(req.stream_id)
                    f.max_concurrent = max(f.max_concurrent, len(f.running))
                time.sleep(f.work)
                with f.lock:
                    f.running.discard(req.stream_id)
                    f.log.append((req.stream_id, req.seq))
                if (req.stream_id, req.seq) in f.fail_run:
                    raise ValueError(f"bad chunk {req.seq}")
                return (req.stream_id, req.seq, req.qp)

            def close(self):
                with f.lock:
                    f.closed.append(sid)
                    f.live_bytes -= self.device_bytes

        s = S()
        with self.lock:
            self.opened.append(sid)
            self.live_bytes += s.device_bytes
            self.max_live_bytes = max(self.max_live_bytes, self.live_bytes)
        return s


def _server(f, slots=4, budget=1e12):
    return ChunkServer(f.open, f.estimate, slots=slots, hbm_budget=budget)


def test_per_stream_order_and_bounded_concurrency():
    f = FakeFactory(work=0.005)
    srv = _server(f, slots=3)
    for sid in range(6):
        srv.open_stream(sid, StreamSpec("enc", 16, 16))
    reqs = [srv.submit(sid, qp, None) for qp in range(5) for sid in range(6)]
    for r in reqs:
        assert r.wait(10) == (r.stream_id, r.seq, r.qp)
    srv.shutdown()
    assert not f.overlap_same_stream
    assert f.max_concurrent == 3  # slots bound the requests in flight
    for sid in range(6):
        assert [q for s, q in f.log if s == sid] == list(range(5))
    assert srv.completed == 30 and srv.failed == 0
    assert sorted(f.closed) == list(range(6))


def test_requests_arriving_later_start_before_earlier_batches_finish():
    """Continuous admission: a request submitted while others run starts when a slot frees,
    before every request submitted earlier has finished."""
    f = FakeFactory(work=0.03)
    srv = _server(f, slots=2)
    for sid in range(3):
        srv.open_stream(sid, StreamSpec("dec", 8, 8))
    first = [srv.submit(0, 1, None) for _ in range(4)]  # a long queue on stream 0
    time.sleep(0.01)
    late = srv.submit(1, 1, None)
    late.wait(10)
    assert not first[-1].finished()
    for r in first:
        r.wait(10)
    srv.shutdown()


def test_admission_waits_for_memory_in_arrival_order():
    f = FakeFactory(work=0.01)
    srv = _server(f, slots=4, budget=2 * 100 * 100)  # room for two 100x100 sessions
    for sid in range(4):
        srv.open_stream(sid, StreamSpec("enc", 100, 100))
    r0 = [srv.submit(0, 0, None) for _ in range(3)]
    r1 = [srv.submit(1, 0, None) for _ in range(3)]
    r2 = srv.submit(2, 0, None)
    r3 = srv.submit(3, 0, None)
    for r in r0 + r1:
        r.wait(10)
    time.sleep(0.05)
    assert not r2.finished() and not r3.finished()  # the budget is held by streams 0 and 1
    assert srv.held_bytes() == 2 * 100 * 100
    srv.close_stream(0)
    r2.wait(10)
    time.sleep(0.05)
    assert not r3.finished()
    srv.close_stream(1)
    r3.wait(10)
    srv.shutdown()
    assert f.opened == [0, 1, 2, 3]
    assert f.max_live_bytes <= 2 * 100 * 100
    assert srv.peak_held <= srv.hbm_budget
    assert srv.held_bytes() == 0


def test_stream_larger_than_budget_is_refused():
    f = FakeFactory()
    srv = _server(f, budget=1000)
    with pytest.raises(ValueError, match="budget"):
        srv.open_stream(0, StreamSpec("enc", 100, 100))
    srv.shutdown()


def test_errors_reach_the_request_and_the_server_keeps_going():
    f = FakeFactory(work=0.001, fail_open={1}, fail_run={(0, 1)})
    srv = _server(f, slots=2)
    srv.open_stream(0, StreamSpec("enc", 8, 8))
    srv.open_stream(1, StreamSpec("enc", 8, 8))
    a = [srv.submit(0, 5, None) for _ in range(3)]
    b = [srv.submit(1, 5, None) for _ in range(2)]
    assert a[0].wait(10) == (0, 0, 5)
    with pytest.raises(ValueError, match="bad chunk 1"):
        a[1].wait(10)
    assert a[2].wait(10) == (0, 2, 5)
    for r in b:
        with pytest.raises(RuntimeError, match="cannot open 1"):
            r.wait(10)
    with pytest.raises(RuntimeError, match="cannot open 1"):
        srv.submit(1, 5, None).wait(10)
    srv.shutdown()
    assert srv.completed == 2 and srv.failed == 4
    assert srv.held_bytes() == 0


def test_submit_validation_and_shutdown_drains():
    f = FakeFactory(work=0.002)
    srv = _server(f, slots=2)
    with pytest.raises(ValueError):
        srv.submit(7, 0, None)
    srv.open_stream(0, StreamSpec("enc", 8, 8))
    with pytest.raises(ValueError):
        srv.open_stream(0, StreamSpec("enc", 8, 8))
    reqs = [srv.submit(0, 0, None) for _ in range(10)]
    srv.shutdown()
    assert all(r.finished() and r.error is None for r in reqs)
    with pytest.raises(ValueError):
        srv.submit(0, 0, None)
    with pytest.raises(ValueError):
        StreamSpec("both", 8, 8)
    with pytest.raises(ValueError):
        StreamSpec("enc", 7, 8)


def test_latency_summary_and_arrivals():
    f = FakeFactory(work=0.002)
    srv = _server(f, slots=2)
    srv.open_stream(0, StreamSpec("enc", 8, 8))
    t0 = time.perf_counter()
    reqs = [srv.submit(0, 0, None, arrival=t0) for _ in range(5)]
    for r in reqs:
        r.wait(10)
    srv.shutdown()
    s = latency_summary(reqs)
    assert s["completed"] == 5 and s["failed"] == 0
    assert 0 < s["p50_ms"] <= s["p99_ms"] <= s["max_ms"]
    lat = sorted(r.latency for r in reqs)
    assert lat[0] >= 0.002  # one chunk of work at least
    rng = np.random.default_rng(0)
    arr = poisson_arrivals(200.0, 5.0, rng)
    assert all(0 < a < 5.0 for a in arr) and arr == sorted(arr)
    assert 850 < len(arr) < 1150


def test_in_flight_limit():
    f = FakeFactory(work=0.02)
    srv = _server(f, slots=4)
    for sid in range(4):
        srv.open_stream(sid, StreamSpec("enc", 8, 8))
    for r in [srv.submit(sid, 0, None) for sid in range(4)]:
        r.wait(10)  # sessions open
    srv.set_in_flight_limit(1)
    f.max_concurrent = 0
    for r in [srv.submit(sid, 0, None) for _ in range(3) for sid in range(4)]:
        r.wait(10)
    assert f.max_concurrent == 1
    srv.set_in_flight_limit(4)
    f.max_concurrent = 0
    for r in [srv.submit(sid, 0, None) for _ in range(3) for sid in range(4)]:
        r.wait(10)
    assert f.max_concurrent == 4
    with pytest.raises(ValueError):
        srv.set_in_flight_limit(5)
    srv.shutdown()


def test_hts_session_bytes_are_the_temporal_context_and_staging():
    """HtsSessionFactory.estimate_bytes: a session holds the stream's temporal context (memory
    and decoded feature 1024 + ctx 512 + I-frame feature 192 channels at 1/8 resolution, 16-bit)
    plus its I420 staging (and an encoder's model-input buffer); the codecs' arenas live in the
    shared pool, not in the sessions."""
    from dcvc_b200.serving import HtsSessionFactory
    f = HtsSessionFactory.__new__(HtsSessionFactory)  # no CUDA needed for the estimate
    ctx = HtsSessionFactory.state_bytes_for(1080, 1920)
    assert ctx == 136 * 240 * 1728 * 2  # ~113 MB at 1080p (padded to 1088)
    planes = 8 * 1080 * 1920 * 3 // 2
    assert f.estimate_bytes(StreamSpec("dec", 1080, 1920)) == ctx + planes
    assert f.estimate_bytes(StreamSpec("enc", 1080, 1920)) == ctx + planes + 8 * 3 * 1080 * 1920 * 2
    assert HtsSessionFactory.state_bytes_for(2160, 3840) == 270 * 480 * 1728 * 2


def test_concurrent_clients_random_work():
    """Four client threads submit to 16 streams at once with random work times, under a budget
    that holds 6 sessions, and close each stream after its last request: every request completes
    in its stream's order, no stream runs two requests at once, and the budget always holds."""
    rng = np.random.default_rng(7)
    works = rng.uniform(0.0, 0.004, size=400)

    class RandFactory(FakeFactory):
        def __init__(self):
            super().__init__(work=0.0)
            self.i = 0

        def open(self, sid, spec):
            s = super().open(sid, spec)
            f = self
            base_run = s.run

            def run(req):
                with f.lock:
                    f.work = float(works[f.i % len(works)])
                    f.i += 1
                return base_run(req)
            s.run = run
            return s

    f = RandFactory()
    srv = _server(f, slots=5, budget=6 * 32 * 32)
    for sid in range(16):
        srv.open_stream(sid, StreamSpec("enc", 32, 32))
    reqs = {sid: [] for sid in range(16)}
    lock = threading.Lock()

    def client(cid):
        for k in range(10):
            for sid in range(cid, 16, 4):
                r = srv.submit(sid, k, None)
                with lock:
                    reqs[sid].append(r)
        for sid in range(cid, 16, 4):
            srv.close_stream(sid)

    threads = [threading.Thread(target=client, args=(c,)) for c in range(4)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    for sid in range(16):
        for k, r in enumerate(reqs[sid]):
            assert r.wait(20) == (sid, k, k)
    srv.shutdown()
    assert not f.overlap_same_stream
    assert f.max_live_bytes <= 6 * 32 * 32 and srv.peak_held <= srv.hbm_budget
    for sid in range(16):
        assert [q for s, q in f.log if s == sid] == list(range(10))
    assert sorted(f.closed) == list(range(16))
    assert srv.held_bytes() == 0 and srv.completed == 160


def test_router_spreads_streams_by_remaining_budget():
    """Streams go to the server with the most budget left after the streams routed to it; their
    requests run there, in order; closing a stream returns its share."""
    from dcvc_b200.serving import StreamRouter
    fa, fb = FakeFactory(work=0.001), FakeFactory(work=0.001)
    a = _server(fa, slots=2, budget=10 * 64 * 64)
    b = _server(fb, slots=2, budget=6 * 64 * 64)
    r = StreamRouter([a, b])
    placed = [r.open_stream(sid, StreamSpec("enc", 64, 64)) for sid in range(8)]
    # each stream takes 1 unit and goes where more units remain after it (a: 10, b: 6; a tie
    # goes to the server with fewer streams): a a a a b a b a
    assert placed == [0, 0, 0, 0, 1, 0, 1, 0]
    reqs = [r.submit(sid, k, None) for k in range(3) for sid in range(8)]
    for q in reqs:
        assert q.wait(10) == (q.stream_id, q.seq, q.qp)
    for sid in range(8):
        f = fa if r.device_of(sid) == 0 else fb
        assert [k for s, k in f.log if s == sid] == [0, 1, 2]
    r.close_stream(0)  # a: 5 units used, b: 2 -> a new stream leaves 4 on a, 3 on b
    assert r.open_stream(100, StreamSpec("enc", 64, 64)) == 0
    with pytest.raises(ValueError):
        r.open_stream(100, StreamSpec("enc", 64, 64))
    with pytest.raises(ValueError, match="budget"):
        r.open_stream(101, StreamSpec("enc", 4096, 4096))
    with pytest.raises(ValueError):
        r.submit(999, 0, None)
    r.shutdown()
    assert a.held_bytes() == 0 and b.held_bytes() == 0
