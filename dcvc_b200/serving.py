"""Continuous-batching chunk server: chunk encode / decode requests of many video streams of mixed
resolution and QP share one GPU.

The reference serves one stream per proxy with one call in flight (a proxy is not re-entrant and
keeps the stream's temporal context inside it, dmc_hts_proxy.h:215-355; the harness walks the
chunks of a sequence one after another, test_video.py:300-345).  This module keeps that contract
per stream and serves many streams at once:

* every stream owns a session (its temporal context in device memory and a CUDA stream; the
  codecs that run its chunks come from a pool shared by all sessions, see HtsSessionFactory);
  the requests of one stream run in arrival order, one at a time;
* `slots` worker threads run the head requests of different streams concurrently, so the kernels
  of one chunk fill the launch gaps, tails and host entropy-coding waits of the others; a request
  that arrives while others are on the GPU starts as soon as a slot frees, not after a batch;
* a stream's session is created when its first request is admitted, and only while the device
  bytes held by all sessions plus the new session's estimate fit the HBM budget; streams waiting
  for memory are admitted strictly in arrival order, and `close_stream` returns a session's
  memory after its last request;
* every request records its arrival, start and completion times (`time.perf_counter`), from
  which `latency_summary` gives throughput and p50 / p99 latency.

The scheduler (`ChunkServer`) knows nothing of CUDA: a session factory supplies sessions with
`run(request)`, `device_bytes` and `close()`.  `HtsSessionFactory` is the HT-S one (enc or dec
role per stream, YUV 4:2:0 planes in and out through host pinned memory).  `StreamRouter` spreads
streams over one server per GPU.
"""
import collections
import threading
import time
from dataclasses import dataclass

import numpy as np

FRAMES = 8  # frames per chunk of the HT-S video model


@dataclass(frozen=True)
class StreamSpec:
    """One video stream: `kind` "enc" (requests carry I420 planes, results are bytes) or "dec"
    (requests carry (bytes, ec_parallel), results are I420 planes) at `height` x `width`."""
    kind: str
    height: int
    width: int

    def __post_init__(self):
        if self.kind not in ("enc", "dec"):
            raise ValueError(f"stream kind must be 'enc' or 'dec', not {self.kind!r}")
        if self.height <= 0 or self.width <= 0 or self.height % 2 or self.width % 2:
            raise ValueError(f"bad stream size {self.height}x{self.width} (positive and even)")


class Request:
    """One chunk request.  `wait()` returns the result or raises the error it failed with."""

    __slots__ = ("stream_id", "qp", "payload", "seq", "arrival", "start", "done", "result",
                 "error", "_event")

    def __init__(self, stream_id, qp, payload, seq, arrival):
        self.stream_id = stream_id
        self.qp = int(qp)
        self.payload = payload
        self.seq = seq            # index of this request within its stream
        self.arrival = arrival
        self.start = None
        self.done = None
        self.result = None
        self.error = None
        self._event = threading.Event()

    def finished(self):
        return self._event.is_set()

    def wait(self, timeout=None):
        if not self._event.wait(timeout):
            raise TimeoutError(f"request {self.seq} of stream {self.stream_id} still pending")
        if self.error is not None:
            raise self.error
        return self.result

    @property
    def latency(self):
        return None if self.done is None else self.done - self.arrival

    def _finish(self, result=None, error=None):
        self.done = time.perf_counter()
        self.result = result
        self.error = error
        self._event.set()


class _Stream:
    __slots__ = ("spec", "session", "pending", "running", "closing", "reserved", "opening",
                 "submitted", "failed_open")

    def __init__(self, spec):
        self.spec = spec
        self.session = None
        self.pending = collections.deque()
        self.running = False
        self.closing = False
        self.reserved = 0      # bytes counted against the budget for this stream
        self.opening = False
        self.submitted = 0
        self.failed_open = None


class ChunkServer:
    """Request loop over per-stream sessions (see the module docstring).

    open_session(stream_id, spec) -> session      called on a worker thread
    estimate_bytes(spec) -> int                   device bytes a new session will hold
    """

    def __init__(self, open_session, estimate_bytes, slots=8, hbm_budget=150e9,
                 on_worker_start=None):
        if slots < 1:
            raise ValueError("slots must be >= 1")
        self._open_session = open_session
        self._estimate = estimate_bytes
        self.hbm_budget = int(hbm_budget)
        self._cv = threading.Condition()
        self._streams = {}
        self._admit_queue = collections.deque()  # streams waiting for a session, in order
        self._held = 0
        self.peak_held = 0
        self.max_sessions = 0
        self.completed = 0
        self.failed = 0
        self._stop = False
        self._limit = slots      # requests in flight at most (<= slots)
        self._in_flight = 0
        self._on_worker_start = on_worker_start
        self._workers = [threading.Thread(target=self._worker, name=f"chunk-slot-{i}", daemon=True)
                         for i in range(slots)]
        for t in self._workers:
            t.start()

    # ------------------------------------------------------------------ client side
    def open_stream(self, stream_id, spec):
        est = int(self._estimate(spec))
        if est > self.hbm_budget:
            raise ValueError(f"stream {stream_id}: a {spec.height}x{spec.width} session needs "
                             f"~{est} device bytes, more than the {self.hbm_budget}-byte budget")
        with self._cv:
            if self._stop:
                raise RuntimeError("server is shut down")
            if stream_id in self._streams:
                raise ValueError(f"stream {stream_id} is already open")
            self._streams[stream_id] = _Stream(spec)

    def submit(self, stream_id, qp, payload, arrival=None):
        """Queues one chunk request of an open stream; `arrival` (perf_counter seconds) defaults
        to now.  Returns the Request."""
        with self._cv:
            st = self._streams.get(stream_id)
            if st is None or st.closing:
                raise ValueError(f"stream {stream_id} is not open")
            if self._stop:
                raise RuntimeError("server is shut down")
            req = Request(stream_id, qp, payload, st.submitted,
                          time.perf_counter() if arrival is None else arrival)
            st.submitted += 1
            if st.failed_open is not None:
                self.failed += 1
                req._finish(error=st.failed_open)
                return req
            st.pending.append(req)
            if st.session is None and not st.opening and stream_id not in self._admit_queue:
                self._admit_queue.append(stream_id)
            self._cv.notify()
            return req

    def close_stream(self, stream_id):
        """The stream's session is released after its queued requests have run."""
        with self._cv:
            st = self._streams.get(stream_id)
            if st is None:
                return
            st.closing = True
            done = self._maybe_release(stream_id, st)
            self._cv.notify_all()
        self._close_all([done])

    def shutdown(self, wait=True):
        """Runs the queued requests, then stops the workers; every stream is closed (idle
        sessions are released at once, which also lets streams waiting for memory in)."""
        done = []
        with self._cv:
            self._stop = True
            for sid in list(self._streams):
                st = self._streams[sid]
                st.closing = True
                done.append(self._maybe_release(sid, st))
            self._cv.notify_all()
        self._close_all(done)
        if wait:
            for t in self._workers:
                t.join()
            done = []
            with self._cv:
                for sid in list(self._streams):
                    st = self._streams[sid]
                    st.closing = True
                    done.append(self._maybe_release(sid, st))
            self._close_all(done)

    def set_in_flight_limit(self, n):
        """Caps the requests in flight at n (1 .. slots); 1 serves one request at a time, as the
        reference's proxies do."""
        n = int(n)
        if not 1 <= n <= len(self._workers):
            raise ValueError(f"in-flight limit must be in 1..{len(self._workers)}")
        with self._cv:
            self._limit = n
            self._cv.notify_all()

    def held_bytes(self):
        with self._cv:
            return self._held

    def sessions(self):
        with self._cv:
            return sum(1 for s in self._streams.values() if s.session is not None)

    # ------------------------------------------------------------------ scheduling
    def _admissible(self, sid):
        """Admission in arrival order: only the first waiting stream may take memory."""
        if not self._admit_queue or self._admit_queue[0] != sid:
            return False
        st = self._streams[sid]
        return self._held + int(self._estimate(st.spec)) <= self.hbm_budget

    def _pick(self):
        """The runnable stream whose head request arrived first, or None."""
        if self._in_flight >= self._limit:
            return None
        best, best_t = None, None
        for sid, st in self._streams.items():
            if st.running or st.opening or not st.pending:
                continue
            if st.session is None and not self._admissible(sid):
                continue
            t = st.pending[0].arrival
            if best is None or t < best_t:
                best, best_t = sid, t
        return best

    def _idle(self):
        return all(not st.pending and not st.running and not st.opening
                   for st in self._streams.values())

    def _maybe_release(self, sid, st):
        """Takes a finished closing stream off the server (call with the lock held).  Returns
        its session, which the caller closes after releasing the lock: closing waits for the
        session's GPU work, and no other slot or client should wait behind that."""
        if st.closing and not st.pending and not st.running and not st.opening:
            session, st.session = st.session, None
            self._held -= st.reserved
            st.reserved = 0
            self._streams.pop(sid, None)
            if sid in self._admit_queue:
                self._admit_queue.remove(sid)
            return session
        return None

    @staticmethod
    def _close_all(sessions):
        for session in sessions:
            if session is not None:
                session.close()

    def _worker(self):
        if self._on_worker_start is not None:
            self._on_worker_start()
        while True:
            with self._cv:
                while True:
                    sid = self._pick()
                    if sid is not None:
                        break
                    if self._stop and self._idle():
                        self._cv.notify_all()
                        return
                    self._cv.wait(0.05)
                st = self._streams[sid]
                need_open = st.session is None
                if need_open:
                    self._admit_queue.popleft()
                    st.reserved = int(self._estimate(st.spec))
                    self._held += st.reserved
                    self.peak_held = max(self.peak_held, self._held)
                    st.opening = True
                else:
                    req = st.pending.popleft()
                    st.running = True
                self._in_flight += 1
            if need_open:
                self._open(sid, st)
                continue
            req.start = time.perf_counter()
            try:
                result = st.session.run(req)
                err = None
            except Exception as e:  # reported through the request
                result, err = None, e
            req._finish(result, err)
            with self._cv:
                st.running = False
                self._in_flight -= 1
                if err is None:
                    self.completed += 1
                else:
                    self.failed += 1
                done = self._maybe_release(sid, st)
                self._cv.notify_all()
            self._close_all([done])

    def _open(self, sid, st):
        try:
            session = self._open_session(sid, st.spec)
            err = None
        except Exception as e:
            session, err = None, e
        with self._cv:
            st.opening = False
            self._in_flight -= 1
            if err is not None:
                # the stream's queued requests fail with the error; its memory is returned
                st.failed_open = err
                self._held -= st.reserved
                st.reserved = 0
                while st.pending:
                    self.failed += 1
                    st.pending.popleft()._finish(error=err)
            else:
                st.session = session
                actual = int(getattr(session, "device_bytes", st.reserved))
                self._held += actual - st.reserved
                st.reserved = actual
                self.peak_held = max(self.peak_held, self._held)
                self.max_sessions = max(self.max_sessions, sum(
                    1 for s in self._streams.values() if s.session is not None))
            done = self._maybe_release(sid, st)
            self._cv.notify_all()
        self._close_all([done])


class StreamRouter:
    """Routes streams over several chunk servers, one per GPU: video streams are independent (a
    stream's temporal context chains only its own chunks), so each stream lives on one device
    and no tensor crosses devices.  A new stream goes to the server with the most budget left
    after the streams already routed to it (their sessions' estimated bytes), ties broken by
    fewer streams; its requests then go where it lives."""

    def __init__(self, servers):
        if not servers:
            raise ValueError("a router needs at least one server")
        self.servers = list(servers)
        self._lock = threading.Lock()
        self._where = {}                      # stream id -> server index
        self._load = [0] * len(self.servers)  # estimated bytes of the streams routed there
        self._count = [0] * len(self.servers)
        self._est = {}

    def open_stream(self, stream_id, spec):
        with self._lock:
            if stream_id in self._where:
                raise ValueError(f"stream {stream_id} is already open")
            ests = [int(srv._estimate(spec)) for srv in self.servers]
            fits = [i for i, srv in enumerate(self.servers) if ests[i] <= srv.hbm_budget]
            if not fits:
                raise ValueError(f"stream {stream_id}: no server's budget holds a "
                                 f"{spec.height}x{spec.width} session")
            best = min(fits, key=lambda i: (-(self.servers[i].hbm_budget - self._load[i] - ests[i]),
                                            self._count[i], i))
            self.servers[best].open_stream(stream_id, spec)
            self._where[stream_id] = best
            self._load[best] += ests[best]
            self._count[best] += 1
            self._est[stream_id] = ests[best]
            return best

    def device_of(self, stream_id):
        with self._lock:
            return self._where[stream_id]

    def submit(self, stream_id, qp, payload, arrival=None):
        with self._lock:
            i = self._where.get(stream_id)
        if i is None:
            raise ValueError(f"stream {stream_id} is not open")
        return self.servers[i].submit(stream_id, qp, payload, arrival)

    def close_stream(self, stream_id):
        with self._lock:
            i = self._where.pop(stream_id, None)
            if i is None:
                return
            self._load[i] -= self._est.pop(stream_id)
            self._count[i] -= 1
        self.servers[i].close_stream(stream_id)

    def shutdown(self, wait=True):
        for srv in self.servers:
            srv.shutdown(wait)


def latency_summary(requests, t0=None):
    """Throughput and latency percentiles of finished requests (seconds -> ms)."""
    done = [r for r in requests if r.done is not None and r.error is None]
    if not done:
        return {"completed": 0, "failed": sum(1 for r in requests if r.error is not None)}
    lat = np.array([r.latency for r in done]) * 1e3
    start = min(r.arrival for r in requests) if t0 is None else t0
    end = max(r.done for r in done)
    return {"completed": len(done),
            "failed": sum(1 for r in requests if r.error is not None),
            "chunks_per_s": round(len(done) / (end - start), 2),
            "p50_ms": round(float(np.percentile(lat, 50)), 2),
            "p99_ms": round(float(np.percentile(lat, 99)), 2),
            "max_ms": round(float(lat.max()), 2)}


def pack_i420(frames, pin=True):
    """List of (y, u, v) uint8 planes -> one uint8 host tensor of the frames' I420 planes back to
    back (the layout of an 8-bit .yuv file), pinned for an asynchronous upload."""
    import torch
    t = torch.from_numpy(np.concatenate(
        [np.concatenate([y.ravel(), u.ravel(), v.ravel()]) for y, u, v in frames]))
    return t.pin_memory() if pin else t


def poisson_arrivals(rate, seconds, rng):
    """Arrival offsets (seconds) of a Poisson process of `rate` per second over `seconds`."""
    out, t = [], 0.0
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= seconds:
            return out
        out.append(t)


class HtsSessionFactory:
    """Sessions of the HT-S chunk codec (DMCHTSProxy) for `ChunkServer`.

    A stream's real state is its temporal context (memory and decoded feature, ctx, the I-frame
    feature: ~113 MB at 1080p), so that is all a session keeps on the device, with its CUDA
    stream and its I420 staging buffers.  The codecs that run the chunks form a pool shared by
    every session of this factory: one parameter set per device (the first codec's set_param,
    the others share_params from it) and per codec one activation arena for one resolution.  A
    request takes an idle codec of its stream's resolution (or creates one; the pool grows to the
    number of requests of each resolution in flight at once, and idle codecs of other resolutions
    are released only beyond `pool_budget` bytes), imports the session's state, codes the chunk,
    exports the state and returns the codec to the pool.  The kernels are deterministic, so a
    stream's results do not depend on which codec ran them.

    A stream is coded in groups of `gop` chunks: the first chunk of every group re-seeds the
    temporal context from the stream's reference frame (the reconstruction of an intra frame in
    the reference's sequence loop, test_video.py:300-320), so a decoder that sees the same group
    of payloads reproduces the encoder's reconstructions.  Encode requests carry the chunk's I420
    planes in host memory (pinned for an asynchronous copy); decode requests carry
    (bytes, ec_parallel) and return the I420 planes in host memory (a fresh copy when
    `copy_output`, else the session's pinned buffer, valid until the stream's next request).
    """

    def __init__(self, state_dict, skip_threshold, ref_frames, gop=2, copy_output=True,
                 device=None, pool_budget=64e9, precision="fp16"):
        import torch
        from .inference_extensions_cuda import DMCHTSProxy
        self._torch = torch
        self.device = torch.cuda.current_device() if device is None else int(device)
        dev = torch.device("cuda", self.device)
        self._refs = {k: v.to(dev) for k, v in ref_frames.items()}  # (H, W) -> [1, 3, Hp, Wp]
        self.gop = int(gop)
        self.copy_output = copy_output
        self.pool_budget = int(pool_budget)
        with torch.cuda.device(dev):
            # this device's own parameter set: sessions never read another GPU's memory
            sd = {k: (v.to(dev) if isinstance(v, torch.Tensor) and v.is_cuda else v)
                  for k, v in state_dict.items()}
            torch.cuda.synchronize(dev)
            self._params = DMCHTSProxy(precision)
            self._params.set_param(sd, skip_threshold)
        self.param_bytes = self._params.stats()[2]
        self._lock = threading.Lock()
        self._free = collections.defaultdict(list)  # (H, W) -> idle codecs, least recent first
        self._codec_bytes = {}                      # (H, W) -> activation bytes of one codec
        self.pool_bytes = 0                         # activation bytes of the live codecs
        self.peak_pool_bytes = 0
        self.codecs_created = 0
        self.codecs_evicted = 0

    def worker_start(self):
        self._torch.cuda.set_device(self.device)

    @staticmethod
    def state_bytes_for(height, width):
        hp, wp = (height + 15) // 16 * 16, (width + 15) // 16 * 16
        return (hp // 8) * (wp // 8) * (1024 + 512 + 192) * 2

    def estimate_bytes(self, spec):
        """Device bytes a session holds: its temporal context plus its I420 staging (and, for an
        encoder, its model-input buffer)."""
        n = FRAMES * spec.height * spec.width * 3 // 2
        extra = n + (FRAMES * 3 * spec.height * spec.width * 2 if spec.kind == "enc" else 0)
        return self.state_bytes_for(spec.height, spec.width) + extra

    def open(self, stream_id, spec):
        return _HtsSession(self, spec)

    # ---- the codec pool
    def _acquire(self, H, W, stream):
        """An idle codec of this resolution, else a new one (sharing the parameters).  A codec
        keeps its arena and its captured phase graphs between requests, so the pool grows to
        the concurrency each resolution sees and stays there; idle codecs of other resolutions
        are released only when the pool would exceed `pool_budget` bytes."""
        from .inference_extensions_cuda import DMCHTSProxy
        torch = self._torch
        key = (H, W)
        evicted = []
        with self._lock:
            if self._free[key]:
                return self._free[key].pop()
            need = self._codec_bytes.get(key, 0)
            while self.pool_bytes + need > self.pool_budget:
                victim = next((k for k, lst in self._free.items() if lst and k != key), None)
                if victim is None:
                    break  # everything else is in use: the budget is exceeded for this request
                evicted.append(self._free[victim].pop(0))
                self.pool_bytes -= self._codec_bytes[victim]
                self.codecs_evicted += 1
            self.codecs_created += 1
        del evicted  # their arenas are freed with them
        codec = DMCHTSProxy(self._params.precision)
        codec.share_params_from(self._params)
        # size the arena for this resolution (the session's state is imported right after)
        with torch.cuda.stream(stream):
            codec.add_ref_feature_from_frame(self._refs[key], False)
        b = codec.stats()[2] - self.param_bytes
        with self._lock:
            self._codec_bytes[key] = b
            self.pool_bytes += b
            self.peak_pool_bytes = max(self.peak_pool_bytes, self.pool_bytes)
        return codec

    def _release(self, H, W, codec):
        with self._lock:
            self._free[(H, W)].append(codec)


class _HtsSession:
    def __init__(self, factory, spec):
        import torch
        from . import ops
        from .synthetic import padding_for
        self._torch, self._ops = torch, ops
        self.factory = factory
        self.spec = spec
        self.gop = factory.gop
        self.copy_output = factory.copy_output
        H, W = spec.height, spec.width
        self.pr, self.pb = padding_for(H, W)
        self.ref = factory._refs[(H, W)]
        dev = torch.device("cuda", factory.device)
        torch.cuda.set_device(dev)
        self.stream = torch.cuda.Stream(device=dev)
        self.count = 0
        n = FRAMES * H * W * 3 // 2
        self.state = torch.empty(factory.state_bytes_for(H, W), dtype=torch.uint8, device=dev)
        self.flags = 0
        self.planes = torch.empty(n, dtype=torch.uint8, device=dev)
        if spec.kind == "enc":
            self.x = torch.empty((1, 3 * FRAMES, H, W), dtype=torch.float16, device=dev,
                                 memory_format=torch.channels_last)
        else:
            self.host_out = torch.empty(n, dtype=torch.uint8).pin_memory()
        self.device_bytes = factory.estimate_bytes(spec)

    def run(self, req):
        torch = self._torch
        H, W = self.spec.height, self.spec.width
        codec = self.factory._acquire(H, W, self.stream)
        try:
            with torch.cuda.stream(self.stream):
                if self.count % self.gop == 0:
                    # a group starts from the reference frame, not from the stored state
                    codec.add_ref_feature_from_frame(self.ref, self.spec.kind == "enc")
                else:
                    codec.import_state(self.state, self.flags)
                self.count += 1
                if self.spec.kind == "enc":
                    planes = req.payload
                    if planes.numel() != self.planes.numel():
                        raise ValueError("encode payload is not 8 I420 frames of the stream's size")
                    self.planes.copy_(planes, non_blocking=True)
                    self._ops.yuv420_to_input(self.planes, FRAMES, H, W, out=self.x)
                    result = codec.compress(self.x, req.qp, False, self.pb, self.pr)
                    _, self.flags = codec.export_state(self.state)
                    return result
                bits, ecp = req.payload
                frames = codec.decompress(bits, req.qp, H, W, ecp, False)
                self._ops.frames_to_yuv420(frames, H, W, out=self.planes)
                _, self.flags = codec.export_state(self.state)
                self.host_out.copy_(self.planes, non_blocking=True)
                self.stream.synchronize()
                return self.host_out.numpy().copy() if self.copy_output else self.host_out
        finally:
            self.factory._release(H, W, codec)

    def close(self):
        self.stream.synchronize()
        self.state = None
