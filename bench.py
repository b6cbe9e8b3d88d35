#!/usr/bin/env python
"""Benchmark of the DCVC-UF HT-S chunk encode+decode hot path on B200.

Workload (one step = one request): one 8-frame 1920x1080 YUV420 chunk (padded to 1920x1088)
compressed by one proxy and decompressed by a second one, QP cycling 0, 21, 42, 63, FP16
activations/weights with FP32 accumulation, synthetic content (dcvc_b200.synthetic), random-init
weights of the HT-S architecture from seed 0 (see `weights` in the JSON config).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl dcvc_b200|reference]

Under torchrun every rank runs its own stream pair on its own GPU (weak scaling, no data-path
collective); the timed region is bracketed by a barrier + device synchronisation and the time is
the maximum over ranks.  `--impl reference` times the reference's CPU path instead (the network
restated on PyTorch CPU in FP32 plus the reference's own rANS coder compiled from its sources) on
the host cores, rank 0 only.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np
import torch

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "1080p YUV420 enc+dec frames/s, batched BF16/FP8 vs plain; p50/p99 chunk latency"
UNIT = "frames/s"
QPS = (0, 21, 42, 63)
FRAMES = 8
SKIP_THRES = 0.15
RESET_INTERVAL = 32  # frames; the reference test harness's default (test_video.py:148)


def reset_at(i):
    """reset_feature_memory of the i-th P chunk of a stream under the reference test harness's
    rule (test_video.py:232-235): chunk i starts at frame 1 + 8 i and resets the temporal memory
    when (frame_idx + 8) % reset_interval == 1, i.e. every fourth chunk at the default 32."""
    return (1 + FRAMES * i + FRAMES) % RESET_INTERVAL == 1
WEIGHTS = ("seed-0 random init of the HT-S architecture (equal to the reference DMC() under "
           "torch.manual_seed(0)), residual-branch output convs scaled x0.1 so activations stay "
           "finite in FP16 (the plain init grows ~1e14x per chunk, in FP64 too)")
PUBLISHED = {"enc_fps_b200": 1415.1, "dec_fps_b200": 945.8, "combined_fps_derived": 567.0}
QUAD_SHAPE = (32640, 1024, 512)  # ffn.0 of a 512-channel dcb2 DepthConvBlock at 1080p


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=4)
    ap.add_argument("--impl", default="dcvc_b200", choices=["dcvc_b200", "reference"])
    ap.add_argument("--height", type=int, default=1080)
    ap.add_argument("--width", type=int, default=1920)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-intra", action="store_true", help="skip the intra-codec measurement")
    ap.add_argument("--no-htl", action="store_true", help="skip the HT-L measurement")
    ap.add_argument("--no-ld", action="store_true", help="skip the low-delay (LD) measurement")
    ap.add_argument("--batch-streams", type=int, default=32,
                    help="streams of the batching form (0 skips it)")
    ap.add_argument("--batch-precision", default="bf16", choices=["fp16", "bf16", "fp8"],
                    help="precision form of the batching form's packed codecs")
    ap.add_argument("--serve-seconds", type=float, default=4.0,
                    help="seconds of Poisson arrivals per offered load of the serving form "
                         "(0 skips it)")
    ap.add_argument("--serve-loads", default="60,120,240",
                    help="offered loads of the serving form, chunks/s")
    ap.add_argument("--serve-streams", type=int, default=24,
                    help="streams of the serving form (half encoders, half decoders)")
    ap.add_argument("--serve-slots", type=int, default=8,
                    help="requests in flight at once in the serving form")
    return ap.parse_args()


def workload_config(H, W, n):
    return {
        "workload": f"DCVC-UF HT-S {W}x{H} YUV420 8-frame chunk encode+decode, QPs 0/21/42/63 "
                    "one request at a time (plain FP16 form)",
        "model": "DCVC-UF HT-S (DMC, ModelStructure.HTS)",
        "resolution": f"{W}x{H}",
        "chunk_frames": FRAMES,
        "qps": list(QPS),
        "skip_threshold": SKIP_THRES,
        "reset_feature_memory": f"every fourth chunk (reset_interval {RESET_INTERVAL} frames, the reference "
                                "test harness's default rule, test_video.py:232-235)",
        "weights": WEIGHTS,
        "l2": "no flush: every step's working set (weights 162 MB + activations > 1 GB) exceeds the 126 MB L2",
        "global_batch": n,
        "parallelism": f"{n} independent stream(s), one per GPU",
    }


# ----------------------------------------------------------------------------- helpers

def max_over_ranks(value, device):
    """Maximum of a float over all ranks of the default process group (or the value itself
    without one); gloo (CPU tensor) or NCCL (device tensor)."""
    import torch.distributed as dist
    t = torch.tensor([float(value)], device=device, dtype=torch.float64)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""

    QUERY = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    # Started before the warm-up so that nvidia-smi is sampling when the timed region begins;
    # stop() keeps the samples whose nvidia-smi timestamp (host local time) falls inside the
    # windows passed to it.
    def __init__(self, device_index):
        uuid = None
        try:
            uuid = "GPU-" + str(torch.cuda.get_device_properties(device_index).uuid)
        except Exception:
            pass
        cmd = ["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits", "-lms", "50"]
        if uuid:
            cmd += ["-i", uuid]
        self.lines = []
        try:
            import threading
            self.p = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.p = None

    def _read(self):
        import datetime
        for line in self.p.stdout:
            try:
                ts = datetime.datetime.strptime(line.split(",")[0].strip(),
                                                "%Y/%m/%d %H:%M:%S.%f").timestamp()
            except ValueError:
                continue
            self.lines.append((ts, line))

    def wait_first_sample(self, timeout=5.0):
        t0 = time.time()
        while self.p is not None and not self.lines and time.time() - t0 < timeout:
            time.sleep(0.01)

    def stop(self, windows=None):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.t.join(timeout=5)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ts, line in self.lines:
            if windows and not any(a <= ts <= b for a, b in windows):
                continue
            parts = [x.strip() for x in line.split(",")][1:]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        loaded = [s for s in sm if s > 0.5 * max(sm)] or sm
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": max(smax),
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return d["hbm_gbs"], d["bf16_tflops"], "measured"
    except Exception:
        return 6650.0, 1590.0, "fallback"


def profiled_traffic(name):
    """DRAM bytes per launch of a kernel from its committed ncu summary
    (profiles/<name>.md, line `traffic_bytes_per_launch: N`), or None."""
    path = os.path.join(ROOT, "profiles", name + ".md")
    try:
        for line in open(path):
            if line.startswith("traffic_bytes_per_launch:"):
                return int(line.split(":")[1].strip())
    except OSError:
        pass
    return None


def _time_rotating(stream, launches, reps=60):
    """Average device time of `launches` (callables over independent operand sets, cycled so
    that consecutive launches read different buffers whose sum exceeds the L2) on `stream`, CUDA
    events around `reps` launches after a warm-up."""
    with torch.cuda.stream(stream):
        for i in range(2 * len(launches)):
            launches[i % len(launches)]()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for i in range(reps):
            launches[i % len(launches)]()
        e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1) / 1e3 / reps


def roofline(stream):
    """The two largest kernels of the 1080p chunk, timed standalone on their launching stream
    with CUDA events at their 1080p shapes and the library's own choice of kernel form:
    the residual GEMM (dc.3 / ffn.2 of a 512-channel block, M=32640 N=512 K=256 + residual;
    HBM-bound, the largest share of the chunk in the launch list) and the quad GEMM (ffn.0 +
    WSiLU chunk-add, M=32640 N=1024 K=512; tensor-bound).  Operand sets rotate through more
    than the 126 MB L2, so inputs come from HBM.  Returns (dominant, [others])."""
    from dcvc_b200 import _native as N, ops
    hbm, peak_tf, kind = measured_peaks()
    g = torch.Generator(device="cuda").manual_seed(7)
    M = QUAD_SHAPE[0]

    def rnd(*shape, scale=1.0):
        return (torch.randn(*shape, device="cuda", generator=g) * scale).half()

    # residual GEMM: three operand sets of 83.5 MB
    res_launch = []
    for _ in range(3):
        a, w = rnd(M, 256), rnd(512, 256, scale=256 ** -0.5)
        r, o = rnd(M, 512), torch.empty(M, 512, device="cuda", dtype=torch.float16)
        b = torch.zeros(512, device="cuda")
        res_launch.append(lambda a=a, w=w, b=b, r=r, o=o: ops.conv1x1(a, w, b, N.EPI_BIAS_RES, res=r, out=o))
    sec = _time_rotating(stream, res_launch)
    byts = (M * 256 + 512 * 256 + 2 * M * 512) * 2
    res = {"kernel": "gemm_stream_kernel<half, res> (dc.3 / ffn.2 + bias + residual, M=32640 N=512 "
                     "K=256; the streaming form the library picks for these shapes)",
           "bound": "hbm", "achieved": round(byts / sec / 1e9, 1), "peak": hbm, "unit": "GB/s",
           "frac": round(byts / sec / 1e9 / hbm, 3), "peak_kind": f"{kind} HBM copy",
           "us_per_launch": round(sec * 1e6, 2), "bytes_per_launch": byts,
           "traffic": profiled_traffic("gemm_res_stream_1080p")}
    # quad GEMM: three operand sets (A 33.4 MB + out 16.7 MB each, plus the 1 MB weights)
    quad_launch = []
    for _ in range(3):
        a, w = rnd(M, 512), rnd(1024, 512, scale=512 ** -0.5)
        o = torch.empty(M, 256, device="cuda", dtype=torch.float16)
        b = torch.zeros(1024, device="cuda")
        quad_launch.append(lambda a=a, w=w, b=b, o=o: ops.conv1x1(a, w, b, N.EPI_QUAD, out=o))
    sec = _time_rotating(stream, quad_launch)
    flops = 2.0 * M * 1024 * 512
    quad = {"kernel": "gemm_sm100_kernel<half, 256, quad> (ffn.0 + WSiLU chunk-add, M=32640 N=1024 K=512)",
            "bound": "tensor", "achieved": round(flops / sec / 1e12, 1), "peak": peak_tf,
            "unit": "TFLOP/s", "frac": round(flops / sec / 1e12 / peak_tf, 3),
            "peak_kind": f"{kind} bf16 burst", "us_per_launch": round(sec * 1e6, 2),
            "flops_per_launch": flops, "traffic": profiled_traffic("gemm_quad_1080p")}
    return res, [quad]


class ReferenceCpuPath:
    """The reference's CPU path for this workload, built without this package's native library:
    the HT-S proxy dataflow restated on PyTorch CPU in FP32 (oracle/hts_oracle.py) and the
    reference's own rANS coder compiled from its sources (oracle/_ref/librans_ref.so).  The CDF
    tables are quantised by the reference's compiled MLCodec_extensions_cpp module
    (oracle/_ref), or, where that module is absent, taken from the reference's own tables
    committed as a fixture (tests/golden/cdf_tables.npz); nothing here loads libdcvc_b200.so.

    One chunk = the full H x W 8-frame chunk compressed by one instance and decompressed by a
    second one, QP cycling as in the GPU arm."""

    def __init__(self, H, W, threads=None):
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import hts_oracle
        from dcvc_b200 import synthetic
        from dcvc_b200.model_spec import calibrated_hts_state_dict
        hts_oracle.use_reference_coder(True)
        self.threads = threads or os.cpu_count() or 1
        torch.set_num_threads(self.threads)
        sd = calibrated_hts_state_dict(0)
        sd, self.tables = _reference_cdf_tables(sd)
        sd = {k: (v.half() if v.is_floating_point() else v) for k, v in sd.items()}
        self.H, self.W = H, W
        self.enc = hts_oracle.HtsOracle(sd, SKIP_THRES, torch.float32)
        self.dec = hts_oracle.HtsOracle(sd, SKIP_THRES, torch.float32)
        ref = synthetic.padded_reference_frame(synthetic.video_chunk_yuv420(2, H, W, 1, 0)[0],
                                               device="cpu")
        self.enc.add_ref_feature_from_frame(ref, True)
        self.dec.add_ref_feature_from_frame(ref, False)
        self.pr, self.pb = synthetic.padding_for(H, W)
        self.xs = [synthetic.to_model_input(synthetic.video_chunk_yuv420(2, H, W, FRAMES, FRAMES * k),
                                            device="cpu") for k in range(2)]
        self.coder = "reference rANS coder compiled from the reference sources"

    def chunk(self, i):
        qp = QPS[i % len(QPS)]
        r = self.enc.compress(self.xs[i % 2], qp, reset_at(i), self.pb, self.pr)
        self.dec.decompress(r["bit_stream"], qp, self.H, self.W, r["ec_parallel"], reset_at(i))
        return r["bit_stream"].size

    def describe(self):
        return (f"full {self.W}x{self.H} 8-frame chunks enc+dec, FP32 PyTorch CPU network on "
                f"{self.threads} threads + {self.coder}; CDF tables: {self.tables}")


def _reference_cdf_tables(sd):
    """Adds the CDF tables with the reference's own quantiser (see ReferenceCpuPath)."""
    ref_dir = os.path.join(ROOT, "oracle", "_ref")
    try:
        sys.path.insert(0, ref_dir)
        import importlib
        ref_mod = importlib.import_module("MLCodec_extensions_cpp")
        if not os.path.abspath(ref_mod.__file__).startswith(ref_dir):
            raise ImportError("not the reference build")
        from dcvc_b200.entropy_tables import add_cdf_to_state_dict
        return (add_cdf_to_state_dict(sd, quantize=ref_mod.pmf_to_quantized_cdf),
                "quantised by the reference's compiled pmf_to_quantized_cdf")
    except ImportError:
        g = np.load(os.path.join(ROOT, "tests", "golden", "cdf_tables.npz"))
        out = dict(sd)
        out["gaussian_encoder.quantized_cdf"] = torch.from_numpy(g["qy"])
        out["gaussian_encoder.cdf_length"] = torch.from_numpy(g["ly"])
        out["bit_estimator_z.quantized_cdf"] = torch.from_numpy(g["qz"])
        out["bit_estimator_z.cdf_length"] = torch.from_numpy(g["lz"])
        return out, "the reference model's own tables (fixture)"
    finally:
        if ref_dir in sys.path:
            sys.path.remove(ref_dir)


def cpu_baseline(H, W, chunks=2):
    """The reference's CPU path (ReferenceCpuPath) on all host cores, timed over `chunks` whole
    H x W chunks after one untimed chunk (a bounded sample of the workload, not scaled)."""
    path = ReferenceCpuPath(H, W)
    path.chunk(0)
    t0 = time.perf_counter()
    for k in range(chunks):
        path.chunk(1 + k)
    sec = time.perf_counter() - t0
    return {"value": round(FRAMES * chunks / sec, 4), "unit": UNIT, "cores": path.threads,
            "kind": "port",
            "sample": f"{chunks} {path.describe()}; {sec:.1f} s timed after one untimed chunk"}


def precision_forms(stream, H, W, xs, steps, warmup, forms=("bf16", "fp8")):
    """The headline workload (one 8-frame chunk compressed and decompressed per step, QPs cycling
    0/21/42/63, inputs resident) in the other precision forms, device-timed like `value`."""
    from dcvc_b200 import synthetic
    from dcvc_b200.entropy_tables import add_cdf_to_state_dict
    from dcvc_b200.inference_extensions_cuda import DMCHTSProxy
    from dcvc_b200.model_spec import calibrated_hts_state_dict
    sd = add_cdf_to_state_dict(calibrated_hts_state_dict(0))
    sd = {k: (v.half().cuda() if v.is_floating_point() else v) for k, v in sd.items()}
    pr, pb = synthetic.padding_for(H, W)
    ref = synthetic.padded_reference_frame(synthetic.video_chunk_yuv420(2, H, W, 1, 0)[0])
    out = {}
    for form in forms:
        enc, dec = DMCHTSProxy(form), DMCHTSProxy(form)
        enc.set_param(sd, SKIP_THRES)
        dec.set_param(sd, SKIP_THRES)
        enc.add_ref_feature_from_frame(ref, True)
        dec.add_ref_feature_from_frame(ref, False)
        nbytes = []

        def step(i):
            qp = QPS[i % len(QPS)]
            bits, ecp = enc.compress(xs[i % 2], qp, reset_at(i), pb, pr)
            dec.decompress(bits, qp, H, W, ecp, reset_at(i))
            nbytes.append(bits.size)

        with torch.cuda.stream(stream):
            for i in range(warmup):
                step(i)
            torch.cuda.synchronize()
            nbytes.clear()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for i in range(steps):
                step(warmup + i)
            e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        out[form] = {"value": round(FRAMES * steps / (ms / 1e3), 2), "unit": UNIT,
                     "ms_per_step": round(ms / steps, 3), "bytes_per_chunk": int(np.mean(nbytes))}
        del enc, dec
    return out


def parity_vs_fp64_oracle(H, W, forms=("fp16", "bf16", "fp8")):
    """Error of every precision form against the FP64 oracle (oracle/hts_oracle.py on the host
    cores) on the benchmark's workload: from one reference frame, the four chunks with QPs
    0/21/42/63 in order, independent temporal state on each side.  Per QP and form: PSNR delta
    (mean over the 8 frames, (6Y+U+V)/8), payload-size delta in percent, fraction of quantised
    latents equal to the oracle's, and whether the decoder reproduced the encoder's symbols
    exactly."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import hts_oracle
    from dcvc_b200 import synthetic
    from dcvc_b200.entropy_tables import add_cdf_to_state_dict
    from dcvc_b200.inference_extensions_cuda import DMCHTSProxy
    from dcvc_b200.model_spec import calibrated_hts_state_dict
    torch.set_num_threads(os.cpu_count() or 1)
    sd = add_cdf_to_state_dict(calibrated_hts_state_dict(0))
    sd = {k: (v.half() if v.is_floating_point() else v) for k, v in sd.items()}
    sd_dev = {k: (v.cuda() if v.is_floating_point() else v) for k, v in sd.items()}
    pr, pb = synthetic.padding_for(H, W)
    ref_frame = synthetic.video_chunk_yuv420(2, H, W, 1, 0)[0]
    chunks = [synthetic.video_chunk_yuv420(2, H, W, FRAMES, FRAMES * k) for k in range(len(QPS))]

    def psnr(xs, frames):
        return float(np.mean([hts_oracle.psnr_yuv420(xs[i].float().cpu(), *frames[i])[0]
                              for i in range(len(frames))]))

    t0 = time.perf_counter()
    oe = hts_oracle.HtsOracle(sd, SKIP_THRES, torch.float64)
    od = hts_oracle.HtsOracle(sd, SKIP_THRES, torch.float64)
    ref_cpu = synthetic.padded_reference_frame(ref_frame, device="cpu")
    oe.add_ref_feature_from_frame(ref_cpu, True)
    od.add_ref_feature_from_frame(ref_cpu, False)
    oracle = []
    for qp, frames in zip(QPS, chunks):
        r = oe.compress(synthetic.to_model_input(frames, device="cpu"), qp, False, pb, pr)
        d = od.decompress(r["bit_stream"], qp, H, W, r["ec_parallel"], False)
        oracle.append((r["bit_stream"].size, psnr(d["x_hat"], frames),
                       r["y_q"][0].permute(1, 2, 0).reshape(-1, 256).float()))
    oracle_s = time.perf_counter() - t0
    out = {"oracle": "FP64 restatement of the HT-S proxy dataflow on the host cores",
           "oracle_seconds": round(oracle_s, 1), "qps": list(QPS), "forms": {}}
    for form in forms:
        enc, dec = DMCHTSProxy(form), DMCHTSProxy(form)
        enc.set_param(sd_dev, SKIP_THRES)
        dec.set_param(sd_dev, SKIP_THRES)
        ref = synthetic.padded_reference_frame(ref_frame)
        enc.add_ref_feature_from_frame(ref, True)
        dec.add_ref_feature_from_frame(ref, False)
        rows = []
        for (qp, frames), (ob, po, oq) in zip(zip(QPS, chunks), oracle):
            bits, ecp = enc.compress(synthetic.to_model_input(frames), qp, False, pb, pr)
            x_hat = dec.decompress(bits, qp, H, W, ecp, False)
            torch.cuda.synchronize()
            exact = all(torch.equal(enc.buffer(n).view(torch.int16), dec.buffer(n).view(torch.int16))
                        for n in ("common", "y_q", "y_hat"))
            agree = float((enc.buffer("y_q").float().cpu() == oq).float().mean())
            rows.append({"qp": qp, "dpsnr_db": round(psnr(x_hat, frames) - po, 4),
                         "dbpp_pct": round(100.0 * (bits.size - ob) / ob, 3),
                         "latent_agree": round(agree, 5), "round_trip_exact": exact})
        out["forms"][form] = rows
        del enc, dec
    return out


def batched_form(args):
    """The batching form: `args.batch_streams` streams (32 by default) of two chunks each, with
    resolutions drawn from seed 3 uniformly over 416x240 .. 3840x2160 and QPs uniform over 0..63.
    Batched: the streams of each resolution form one packed batch (DMCHTSProxy.compress_batch /
    decompress_batch, BF16 form), so every network layer is one launch over all streams of that
    resolution; the resolution groups run concurrently, one host thread and CUDA stream each.
    Plain: the same chunks coded one request at a time by single-stream FP16 codecs (the
    reference's form).  Both encode and decode every chunk; both are device-timed from one start
    event to one end event.  Reported in frames/s and 1080p-equivalent frames/s (pixels)."""
    import threading
    from dcvc_b200 import synthetic
    from dcvc_b200.entropy_tables import add_cdf_to_state_dict
    from dcvc_b200.inference_extensions_cuda import DMCHTSProxy
    from dcvc_b200.model_spec import calibrated_hts_state_dict
    rng = np.random.default_rng(3)
    n = args.batch_streams
    sizes = [SERVE_SIZES[i] for i in rng.integers(0, len(SERVE_SIZES), size=n)]
    qps = [[int(q) for q in rng.integers(0, 64, size=2)] for _ in range(n)]
    sd = add_cdf_to_state_dict(calibrated_hts_state_dict(0))
    sd = {k: (v.half().cuda() if v.is_floating_point() else v) for k, v in sd.items()}
    groups = {}
    for i, s in enumerate(sizes):
        groups.setdefault(s, []).append(i)
    refs = [synthetic.padded_reference_frame(synthetic.video_chunk_yuv420(100 + i, *sizes[i], 1, 0)[0])
            for i in range(n)]
    xs = [[synthetic.to_model_input(synthetic.video_chunk_yuv420(100 + i, *sizes[i], FRAMES, FRAMES * c))
           for c in range(2)] for i in range(n)]
    px = sum(h * w for h, w in sizes) * 2 * FRAMES
    frames = n * 2 * FRAMES

    def proxies(form):
        enc, dec = DMCHTSProxy(form), DMCHTSProxy(form)
        enc.set_param(sd, SKIP_THRES)
        dec.set_param(sd, SKIP_THRES)
        return enc, dec

    # ---- batched: one packed enc/dec pair per resolution group, groups concurrently
    work = []
    for (h, w), ids in sorted(groups.items()):
        enc, dec = proxies(args.batch_precision)
        work.append({"hw": (h, w), "ids": ids, "enc": enc, "dec": dec, "stream": torch.cuda.Stream(),
                     "err": None})

    def run_group(g, seed_only=False):
        h, w = g["hw"]
        pr, pb = synthetic.padding_for(h, w)
        ids = g["ids"]
        with torch.cuda.stream(g["stream"]):
            g["enc"].add_ref_features_from_frames([refs[i] for i in ids], True)
            g["dec"].add_ref_features_from_frames([refs[i] for i in ids], False)
            if seed_only:
                return
            for c in range(2):
                q = [qps[i][c] for i in ids]
                out = g["enc"].compress_batch([xs[i][c] for i in ids], q, False, pb, pr)
                g["dec"].decompress_batch([b for b, _ in out], q, h, w, [e for _, e in out], False)

    def timed(groups_, fn):
        start_stream = torch.cuda.Stream()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(start_stream)
        errors = []

        def body(g):
            try:
                g["stream"].wait_event(e0)
                fn(g)
            except Exception as ex:  # noqa: BLE001
                errors.append(f"{type(ex).__name__}: {ex}")

        th = [threading.Thread(target=body, args=(g,)) for g in groups_]
        for t in th:
            t.start()
        for t in th:
            t.join()
        for g in groups_:
            start_stream.wait_stream(g["stream"])
        e1.record(start_stream)
        e1.synchronize()
        if errors:
            raise RuntimeError(errors[0])
        return e0.elapsed_time(e1) / 1e3

    for _ in range(2):  # warm-up: sizes the arenas, captures the phase graphs
        timed(work, run_group)
    sec_b = timed(work, run_group)
    launches = sum(g["enc"].stats()[1] + g["dec"].stats()[1] for g in work)
    for g in work:
        g["enc"] = g["dec"] = None
    del work
    torch.cuda.empty_cache()

    # ---- plain: the same chunks one request at a time, single-stream FP16 codecs
    plain = {}
    for hw in sorted(groups):
        plain[hw] = proxies("fp16")

    def run_plain(g):
        for i in range(n):
            h, w = sizes[i]
            pr, pb = synthetic.padding_for(h, w)
            enc, dec = plain[(h, w)]
            enc.add_ref_feature_from_frame(refs[i], True)
            dec.add_ref_feature_from_frame(refs[i], False)
            for c in range(2):
                bits, ecp = enc.compress(xs[i][c], qps[i][c], False, pb, pr)
                dec.decompress(bits, qps[i][c], h, w, ecp, False)

    one = [{"stream": torch.cuda.Stream()}]

    def plain_body(g):
        with torch.cuda.stream(g["stream"]):
            run_plain(g)

    timed(one, plain_body)  # warm-up
    sec_p = timed(one, plain_body)
    eq = px / (1920 * 1080)
    return {"streams": n, "chunks_per_stream": 2, "precision": args.batch_precision,
            "streams_by_size": {f"{w}x{h}": len(ids) for (h, w), ids in sorted(groups.items())},
            "batched": {"frames_per_s": round(frames / sec_b, 1),
                        "frames_1080p_equiv_per_s": round(eq / sec_b, 1),
                        "seconds": round(sec_b, 4), "launches_last_call": launches},
            "plain_fp16": {"frames_per_s": round(frames / sec_p, 1),
                           "frames_1080p_equiv_per_s": round(eq / sec_p, 1),
                           "seconds": round(sec_p, 4)},
            "batched_vs_plain": round(sec_p / sec_b, 3),
            "note": "packed batches per resolution group (one launch per layer over the group's "
                    "streams), groups concurrent; each stream's bytes equal its single-stream "
                    "coding (tests/test_batch_gpu.py); random-init weights, synthetic content"}


SERVE_SIZES = ((240, 416), (480, 832), (720, 1280), (1080, 1920), (2160, 3840))
SERVE_WEIGHTS = (0.10, 0.20, 0.30, 0.30, 0.10)
SERVE_BUDGET = 150e9


def serving_bench(args):
    """The serving form: Poisson arrivals of chunk encode and decode requests (50/50) at each
    offered load, over a fixed set of streams whose resolutions are drawn with the weights
    10/20/30/30/10 % over 416x240 .. 3840x2160 (seed 3), QP uniform over 0..63, through the
    continuous-batching ChunkServer (per-stream temporal context resident in HBM, admission by
    a 150 GB budget, host rANS of one request overlapping the GPU work of the others).

    Encode requests carry the chunk's 8-bit I420 planes from pinned host memory and return the
    payload bytes; decode requests carry payload bytes and return the I420 planes in pinned host
    memory, so every request is end to end.  A stream codes groups of two chunks, re-seeding its
    temporal context at each group start, so decoders replay the two pre-encoded payloads of
    their group.  Latency = completion - scheduled arrival (host clock, as a client sees it)."""
    from dcvc_b200 import synthetic
    from dcvc_b200.entropy_tables import add_cdf_to_state_dict
    from dcvc_b200.model_spec import calibrated_hts_state_dict
    from dcvc_b200.serving import (ChunkServer, HtsSessionFactory, StreamSpec, latency_summary,
                                   pack_i420, poisson_arrivals)
    rng = np.random.default_rng(3)
    n_enc = args.serve_streams // 2
    n_dec = args.serve_streams - n_enc
    pick = rng.choice(len(SERVE_SIZES), size=args.serve_streams, p=SERVE_WEIGHTS)
    sizes = [SERVE_SIZES[i] for i in pick]
    used = sorted(set(sizes))
    content = {s: [pack_i420(synthetic.video_chunk_yuv420(2, s[0], s[1], FRAMES, FRAMES * k))
                   for k in range(2)] for s in used}
    refs = {s: synthetic.padded_reference_frame(synthetic.video_chunk_yuv420(2, s[0], s[1], 1, 0)[0])
            for s in used}
    sd = add_cdf_to_state_dict(calibrated_hts_state_dict(0))
    sd = {k: (v.half().cuda() if v.is_floating_point() else v) for k, v in sd.items()}
    torch.cuda.synchronize()
    f = HtsSessionFactory(sd, SKIP_THRES, refs, gop=2, copy_output=False)
    srv = ChunkServer(f.open, f.estimate_bytes, slots=args.serve_slots, hbm_budget=SERVE_BUDGET,
                      on_worker_start=f.worker_start)
    try:
        enc_ids = [f"enc{i}" for i in range(n_enc)]
        dec_ids = [f"dec{i}" for i in range(n_dec)]
        spec = {}
        for i, sid in enumerate(enc_ids + dec_ids):
            spec[sid] = StreamSpec("enc" if sid.startswith("enc") else "dec", *sizes[i])
        # decoders' payloads: one group of two chunks per decoder at its own QPs
        dec_qps = {sid: [int(q) for q in rng.integers(0, 64, size=2)] for sid in dec_ids}
        payloads = {}
        for sid in dec_ids:
            pre = "pre-" + sid
            srv.open_stream(pre, StreamSpec("enc", spec[sid].height, spec[sid].width))
            s = (spec[sid].height, spec[sid].width)
            rs = [srv.submit(pre, dec_qps[sid][k], content[s][k]) for k in range(2)]
            payloads[sid] = [r.wait(600) for r in rs]
            srv.close_stream(pre)
        # open the streams and run one group each (sessions created, graphs captured)
        for sid in enc_ids + dec_ids:
            srv.open_stream(sid, spec[sid])
        # streams of one resolution back to back, so that the warm-up reaches the largest number
        # of same-resolution requests in flight that the loads can reach and the codec pool is
        # grown (arenas allocated, graphs captured) before any timed load
        warm = []
        by_size = sorted(enc_ids + dec_ids, key=lambda i: (spec[i].height, spec[i].width, i))
        for k in range(2):
            for sid in by_size:
                if sid in payloads:
                    warm.append(srv.submit(sid, dec_qps[sid][k], payloads[sid][k]))
                else:
                    s = (spec[sid].height, spec[sid].width)
                    warm.append(srv.submit(sid, int(rng.integers(0, 64)), content[s][k]))
        for r in warm:
            r.wait(600)
        nxt = {sid: 2 for sid in enc_ids + dec_ids}

        def draw(times):
            """(arrival offset, stream, qp, payload) per arrival: encode or decode 50/50."""
            plan = []
            for t in times:
                if rng.random() < 0.5:
                    sid = enc_ids[int(rng.integers(0, n_enc))]
                    s = (spec[sid].height, spec[sid].width)
                    plan.append((t, sid, int(rng.integers(0, 64)), content[s][nxt[sid] % 2]))
                else:
                    sid = dec_ids[int(rng.integers(0, n_dec))]
                    k = nxt[sid] % 2
                    plan.append((t, sid, dec_qps[sid][k], payloads[sid][k]))
                nxt[sid] += 1
            return plan

        def run_plan(plan):
            reqs = []
            t0 = time.perf_counter()
            for t, sid, qp, payload in plan:
                delay = t0 + t - time.perf_counter()
                if delay > 0:
                    time.sleep(delay)
                reqs.append(srv.submit(sid, qp, payload, arrival=t0 + t))
            errors = []
            for r in reqs:
                try:
                    r.wait(600)
                except TimeoutError:
                    raise
                except Exception as e:  # counted as failed in the summary; the first is shown
                    errors.append(f"{type(e).__name__}: {e}")
            summ = latency_summary(reqs, t0)
            if errors:
                summ["first_error"] = errors[0][:200]
            ok = [r for r in reqs if r.error is None]
            px = sum(spec[r.stream_id].height * spec[r.stream_id].width for r in ok)
            span = max(r.done for r in reqs) - t0
            summ.update({"requests": len(reqs),
                         "frames_per_s": round(len(ok) * FRAMES / span, 1),
                         "frames_1080p_equiv_per_s": round(px * FRAMES / (1920 * 1080) / span, 1)})
            return summ

        loads = []
        for rate in [float(x) for x in args.serve_loads.split(",") if x]:
            summ = run_plan(draw(poisson_arrivals(rate, args.serve_seconds, rng)))
            summ["offered_chunks_per_s"] = rate
            loads.append(summ)
        # saturation: the same mix with every request queued at once, one request in flight (the
        # plain one-request-at-a-time form) against `slots` in flight
        n_sat = min(480, max(64, int(120 * args.serve_seconds)))
        saturation = {}
        for limit in (1, args.serve_slots):
            srv.set_in_flight_limit(limit)
            # arrival offsets 1 us apart keep the service order first-come first-served
            saturation[f"in_flight_{limit}"] = run_plan(draw([i * 1e-6 for i in range(n_sat)]))
        srv.set_in_flight_limit(args.serve_slots)
        a = saturation[f"in_flight_{args.serve_slots}"]["frames_1080p_equiv_per_s"]
        b = saturation["in_flight_1"]["frames_1080p_equiv_per_s"]
        saturation["speedup"] = round(a / b, 3) if b else None
        streams_by_size = {f"{w}x{h}": sum(1 for s in sizes if s == (h, w)) for h, w in used}
        return {"loads": loads, "saturation": saturation, "streams": args.serve_streams,
                "streams_by_size": streams_by_size,
                "slots": args.serve_slots, "seconds_per_load": args.serve_seconds,
                "hbm_budget_gb": SERVE_BUDGET / 1e9, "peak_held_gb": round(srv.peak_held / 1e9, 2),
                "peak_codec_pool_gb": round(f.peak_pool_bytes / 1e9, 2),
                "param_gb": round(f.param_bytes / 1e9, 3),
                "peak_total_gb": round((srv.peak_held + f.peak_pool_bytes + f.param_bytes) / 1e9, 2),
                "memory_model": "sessions hold only their temporal context and I420 staging "
                                "(peak_held_gb); chunks run on a pool of codecs, as many per "
                                "resolution as its requests in flight at once "
                                "(peak_codec_pool_gb), sharing one parameter set (param_gb)",
                "codecs_created": f.codecs_created, "codecs_evicted": f.codecs_evicted,
                "max_sessions": srv.max_sessions, "failed": srv.failed,
                "note": "Poisson arrivals, 50/50 encode/decode, resolutions 10/20/30/30/10 % over "
                        "416x240..3840x2160, QP U[0,63]; end to end (I420 planes host<->device); "
                        "latency on the host clock from scheduled arrival to result; a request "
                        "codes OR decodes its chunk, so its frames count once"}
    finally:
        srv.shutdown()


def split_enc_dec(enc, dec, xs, args, pb, pr, H, W, stream):
    """Encode-only and decode-only throughput of the same chunks (separate timed loops); the
    decoder replays the payloads recorded by the encoder, so both keep their temporal state in
    step."""
    n = max(4, args.steps)
    payloads = []
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for i in range(n):
        qp = QPS[i % len(QPS)]
        bits, ecp = enc.compress(xs[i % 2], qp, reset_at(i), pb, pr)
        payloads.append((bits, qp, ecp, reset_at(i)))
    e1.record(stream)
    torch.cuda.synchronize()
    enc_ms = e0.elapsed_time(e1)
    e0.record(stream)
    for bits, qp, ecp, reset in payloads:
        dec.decompress(bits, qp, H, W, ecp, reset)
    e1.record(stream)
    torch.cuda.synchronize()
    dec_ms = e0.elapsed_time(e1)
    return {"enc": round(FRAMES * n / (enc_ms / 1e3), 1), "dec": round(FRAMES * n / (dec_ms / 1e3), 1),
            "chunks": n, "note": "device-timed, inputs resident; compare reference_published"}


def htl_bench(stream, H, W, chunks=8, warmup=3):
    """The HT-L model (DMCHTLProxy): encode-only and decode-only frames/s of 1080p chunks, QPs
    cycling as in the main workload; the reference publishes these for B200."""
    from dcvc_b200 import synthetic
    from dcvc_b200.entropy_tables import add_cdf_to_state_dict
    from dcvc_b200.inference_extensions_cuda import DMCHTLProxy
    from dcvc_b200.model_spec import calibrated_htl_state_dict
    sd = add_cdf_to_state_dict(calibrated_htl_state_dict(0))
    sd = {k: (v.half().cuda() if v.is_floating_point() else v) for k, v in sd.items()}
    enc, dec = DMCHTLProxy(), DMCHTLProxy()
    enc.set_param(sd, SKIP_THRES)
    dec.set_param(sd, SKIP_THRES)
    del sd
    ref = synthetic.padded_reference_frame(synthetic.video_chunk_yuv420(2, H, W, 1, 0)[0])
    enc.add_ref_feature_from_frame(ref, True)
    dec.add_ref_feature_from_frame(ref, False)
    pr, pb = synthetic.padding_for(H, W)
    xs = [synthetic.to_model_input(synthetic.video_chunk_yuv420(2, H, W, FRAMES, FRAMES * k))
          for k in range(2)]
    for i in range(warmup):
        qp = QPS[i % len(QPS)]
        bits, ecp = enc.compress(xs[i % 2], qp, reset_at(i), pb, pr)
        dec.decompress(bits, qp, H, W, ecp, reset_at(i))
    torch.cuda.synchronize()
    e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    payloads = []
    e[0].record(stream)
    for i in range(chunks):
        qp = QPS[i % len(QPS)]
        bits, ecp = enc.compress(xs[i % 2], qp, reset_at(i), pb, pr)
        payloads.append((bits, qp, ecp, reset_at(i)))
    e[1].record(stream)
    for bits, qp, ecp, reset in payloads:
        dec.decompress(bits, qp, H, W, ecp, reset)
    e[2].record(stream)
    torch.cuda.synchronize()
    te, td = e[0].elapsed_time(e[1]) / chunks, e[1].elapsed_time(e[2]) / chunks
    return {"enc_fps": round(FRAMES * 1e3 / te, 1), "dec_fps": round(FRAMES * 1e3 / td, 1),
            "enc_ms_per_chunk": round(te, 3), "dec_ms_per_chunk": round(td, 3),
            "bytes_per_chunk": int(np.mean([p[0].size for p in payloads])), "chunks": chunks,
            "reference_published": {"enc_fps_b200": 811.7, "dec_fps_b200": 551.6}}


def ld_bench(stream, H, W, frames=32, warmup=4, reset_interval=8):
    """The low-delay model (DMCLDProxy): encode-only and decode-only frames/s at 1080p, one frame
    per call, QPs cycling as in the main workload; the reference publishes these for B200.  The
    temporal memory is reset with the test harness's rule (test_video.py:232-235,
    (frame_idx + 1) % reset_interval == 1) every 8 frames: the random-init LD recurrence grows its
    latents frame after frame (the bitrate rises 6x over 20 frames), and the reset keeps it at the
    rate of the first frames."""
    from dcvc_b200 import synthetic
    from dcvc_b200.entropy_tables import add_cdf_to_state_dict
    from dcvc_b200.inference_extensions_cuda import DMCLDProxy
    from dcvc_b200.model_spec import calibrated_ld_state_dict
    sd = add_cdf_to_state_dict(calibrated_ld_state_dict(0))
    sd = {k: (v.half().cuda() if v.is_floating_point() else v) for k, v in sd.items()}
    enc, dec = DMCLDProxy(), DMCLDProxy()
    enc.set_param(sd, SKIP_THRES)
    dec.set_param(sd, SKIP_THRES)
    del sd
    yuv = synthetic.video_chunk_yuv420(2, H, W, FRAMES + 1, 0)
    ref = synthetic.padded_reference_frame(yuv[0])
    enc.add_ref_feature_from_frame(ref, True)
    dec.add_ref_feature_from_frame(ref, False)
    pr, pb = synthetic.padding_for(H, W)
    xs = [synthetic.to_model_input([f]) for f in yuv[1:]]

    def reset_at(i):  # frame_idx = i + 1 after the intra frame
        return (i + 2) % reset_interval == 1

    for i in range(warmup):
        qp = QPS[i % len(QPS)]
        bits, ecp = enc.compress(xs[i % len(xs)], qp, reset_at(i), pb, pr)
        dec.decompress(bits, qp, H, W, ecp, reset_at(i))
    torch.cuda.synchronize()
    e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    payloads = []
    e[0].record(stream)
    for i in range(warmup, warmup + frames):
        qp = QPS[i % len(QPS)]
        bits, ecp = enc.compress(xs[i % len(xs)], qp, reset_at(i), pb, pr)
        payloads.append((bits, qp, ecp, reset_at(i)))
    e[1].record(stream)
    for bits, qp, ecp, reset in payloads:
        dec.decompress(bits, qp, H, W, ecp, reset)
    e[2].record(stream)
    torch.cuda.synchronize()
    te, td = e[0].elapsed_time(e[1]) / frames, e[1].elapsed_time(e[2]) / frames
    return {"enc_fps": round(1e3 / te, 1), "dec_fps": round(1e3 / td, 1),
            "enc_ms_per_frame": round(te, 3), "dec_ms_per_frame": round(td, 3),
            "bytes_per_frame": int(np.mean([p[0].size for p in payloads])), "frames": frames,
            "reset_interval": reset_interval,
            "reference_published": {"enc_fps_b200": 625.6, "dec_fps_b200": 621.9}}


def intra_bench(stream, H, W, reps=10):
    """The intra (DMCI) codec: encode-only and decode-only frames/s at the bench resolution and
    at 256x256 (the reference's CPU-runnable intra case), QP 32."""
    from dcvc_b200 import synthetic
    from dcvc_b200.entropy_tables import add_cdf_to_state_dict
    from dcvc_b200.inference_extensions_cuda import DMCIProxy
    from dcvc_b200.model_spec import calibrated_dmci_state_dict
    sd = add_cdf_to_state_dict(calibrated_dmci_state_dict(0))
    sd = {k: (v.half().cuda() if v.is_floating_point() else v) for k, v in sd.items()}
    enc, dec = DMCIProxy(), DMCIProxy()
    enc.set_param(sd, SKIP_THRES)
    dec.set_param(sd, SKIP_THRES)
    out = {}
    for (h, w), key in (((H, W), f"{W}x{H}"), ((256, 256), "256x256")):
        x = synthetic.to_model_input([synthetic.intra_frame_yuv420(1, h, w)])
        pr, pb = synthetic.padding_for(h, w)
        for i in range(3):
            bits, _, ecp = enc.compress(x, 32, pb, pr)
            dec.decompress(bits, 32, h, w, ecp)
        torch.cuda.synchronize()
        e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        e[0].record(stream)
        for i in range(reps):
            bits, _, ecp = enc.compress(x, 32, pb, pr)
        e[1].record(stream)
        for i in range(reps):
            dec.decompress(bits, 32, h, w, ecp)
        e[2].record(stream)
        torch.cuda.synchronize()
        te, td = e[0].elapsed_time(e[1]) / reps, e[1].elapsed_time(e[2]) / reps
        out[key] = {"enc_fps": round(1e3 / te, 1), "dec_fps": round(1e3 / td, 1),
                    "enc_ms": round(te, 3), "dec_ms": round(td, 3), "bytes": int(bits.size)}
    out["qp"] = 32
    out["reference_published"] = "DCVC-UF-Intra 1080p enc/dec 81.5/95.0 frames/s on A100 (README)"
    return out


# ----------------------------------------------------------------------------- arms

def _section(fn, *a):
    """fn(*a), or {"error": ...} when it raises."""
    try:
        return fn(*a)
    except Exception as e:  # noqa: BLE001
        return {"error": f"{type(e).__name__}: {e}"[:300]}


def _empty_cache():
    try:
        torch.cuda.empty_cache()
    except RuntimeError:
        pass  # a context broken by a failed section; the CPU baseline and the line still follow


def run_reference(args):
    """The reference arm: the reference's CPU path (ReferenceCpuPath) on the host cores, one
    whole chunk per step, W untimed and K timed steps, wall clock around each step (there is no
    device work).  Rank 0 alone runs it; under torchrun the other ranks exit at once."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    H, W = args.height, args.width
    path = ReferenceCpuPath(H, W)
    for i in range(args.warmup):
        path.chunk(i)
    per_step = []
    t0 = time.perf_counter()
    for i in range(args.steps):
        t = time.perf_counter()
        path.chunk(args.warmup + i)
        per_step.append(time.perf_counter() - t)
    total = time.perf_counter() - t0
    value = round(FRAMES * args.steps / total, 4)
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "impl": "reference",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(total / args.steps * 1e3, 1), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(H, W, args.gpus),
        "latency_ms": {"p50": round(float(np.percentile(per_step, 50)) * 1e3, 1),
                       "p99": round(float(np.percentile(per_step, 99)) * 1e3, 1)},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": path.threads, "kind": "port",
                         "sample": "every step: one " + path.describe()},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)


def run_gpu(args):
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", local))
    from dcvc_b200 import synthetic
    from dcvc_b200.entropy_tables import add_cdf_to_state_dict
    from dcvc_b200.inference_extensions_cuda import DMCHTSProxy
    from dcvc_b200.model_spec import calibrated_hts_state_dict

    H, W = args.height, args.width
    sd = add_cdf_to_state_dict(calibrated_hts_state_dict(0))
    sd = {k: (v.half().cuda() if v.is_floating_point() else v) for k, v in sd.items()}
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    enc, dec = DMCHTSProxy(), DMCHTSProxy()
    enc.set_param(sd, SKIP_THRES)
    dec.set_param(sd, SKIP_THRES)
    del sd
    # stream content differs per rank
    seed = 2 + rank
    ref = synthetic.padded_reference_frame(synthetic.video_chunk_yuv420(seed, H, W, 1, 0)[0])
    enc.add_ref_feature_from_frame(ref, True)
    dec.add_ref_feature_from_frame(ref, False)
    pr, pb = synthetic.padding_for(H, W)
    host_chunks = [synthetic.video_chunk_yuv420(seed, H, W, FRAMES, FRAMES * k) for k in range(2)]
    xs = [synthetic.to_model_input(c) for c in host_chunks]

    def step(i, x):
        qp = QPS[i % len(QPS)]
        bits, ecp = enc.compress(x, qp, reset_at(i), pb, pr)
        return dec.decompress(bits, qp, H, W, ecp, reset_at(i)), bits.size

    clocks = ClockSampler(local)
    clocks.wait_first_sample()
    for i in range(args.warmup):
        step(i, xs[i % 2])
    torch.cuda.synchronize()

    # ---------------- timed region: inputs resident in HBM
    kernels_per_step = enc.stats()[1] + dec.stats()[1]
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    windows = [[time.time(), None]]
    marks = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    marks[0].record(stream)
    nbytes = []
    for i in range(args.steps):
        _, nb = step(args.warmup + i, xs[i % 2])
        nbytes.append(nb)
        marks[i + 1].record(stream)
    torch.cuda.synchronize()
    windows[-1][1] = time.time()
    if world > 1:
        dist.barrier()
    ms = marks[0].elapsed_time(marks[-1])
    lat = [marks[i].elapsed_time(marks[i + 1]) for i in range(args.steps)]
    ms_max = max_over_ranks(ms, "cuda")
    value = FRAMES * args.steps * world / (ms_max / 1e3)

    # ---------------- end to end through the proxy API from pinned host memory: the chunk's
    # 8-bit YUV 4:2:0 planes go up, are converted to the model input on the device (the FP16
    # arithmetic of get_src_frame), and the 8 reconstructions come back as YUV 4:2:0 planes (the
    # decoded-frame writer of the reference harness).  The copies run on a second stream with
    # double-buffered planes, as a serving loop would: chunk i+1 goes up and chunk i comes back
    # while chunk i+1 is coded; every copy is inside the timed region.
    from dcvc_b200 import ops
    planes_host = [torch.from_numpy(np.concatenate(
        [np.concatenate([y.ravel(), u.ravel(), v.ravel()]) for y, u, v in c])).pin_memory()
        for c in host_chunks]
    planes_dev = [torch.empty_like(planes_host[0], device="cuda") for _ in range(2)]
    out_dev = [torch.empty_like(planes_dev[0]) for _ in range(2)]
    out_host = [torch.empty_like(planes_host[0]).pin_memory() for _ in range(2)]
    x_dev = torch.empty_like(xs[0])
    copy = torch.cuda.Stream()
    ev = {k: [torch.cuda.Event() for _ in range(2)] for k in ("up", "conv", "ready", "down")}
    h2d = planes_host[0].numel()
    d2h = out_host[0].numel()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    windows.append([time.time(), None])
    e0.record(stream)
    copy.wait_event(e0)
    with torch.cuda.stream(copy):
        planes_dev[0].copy_(planes_host[0], non_blocking=True)
        ev["up"][0].record(copy)
    for i in range(args.steps):
        b, nb = i % 2, (i + 1) % 2
        if i + 1 < args.steps:
            with torch.cuda.stream(copy):
                if i >= 1:
                    copy.wait_event(ev["conv"][nb])  # chunk i-1 has been converted
                planes_dev[nb].copy_(planes_host[(i + 1) % 2], non_blocking=True)
                ev["up"][nb].record(copy)
        stream.wait_event(ev["up"][b])
        ops.yuv420_to_input(planes_dev[b], FRAMES, H, W, out=x_dev)
        ev["conv"][b].record(stream)
        frames, _ = step(args.warmup + i, x_dev)
        if i >= 2:
            stream.wait_event(ev["down"][b])  # chunk i-2 has been read back
        ops.frames_to_yuv420(frames, H, W, out=out_dev[b])
        ev["ready"][b].record(stream)
        with torch.cuda.stream(copy):
            copy.wait_event(ev["ready"][b])
            out_host[b].copy_(out_dev[b], non_blocking=True)
            ev["down"][b].record(copy)
    for k in range(min(2, args.steps)):
        stream.wait_event(ev["down"][(args.steps - 1 - k) % 2])
    e1.record(stream)
    torch.cuda.synchronize()
    windows[-1][1] = time.time()
    e2e = FRAMES * args.steps * world / (max_over_ranks(e0.elapsed_time(e1), "cuda") / 1e3)

    # ---------------- encode alone and decode alone (the reference publishes them separately)
    split = split_enc_dec(enc, dec, xs, args, pb, pr, H, W, stream)
    # ---------------- the same workload in the BF16 and FP8 precision forms
    forms = _section(precision_forms, stream, H, W, xs, args.steps, args.warmup)
    clk = clocks.stop(windows)
    roof, roof_others = roofline(stream)
    # The extra measurements below report a failure in their own key instead of losing the line
    # (and every rank still reaches the closing barrier).
    intra = None if args.no_intra else _section(intra_bench, stream, H, W)
    htl = None if args.no_htl else _section(htl_bench, stream, H, W)
    ld = None if args.no_ld else _section(ld_bench, stream, H, W)
    del enc, dec
    _empty_cache()
    batched = _section(batched_form, args) if args.batch_streams > 0 else None
    _empty_cache()
    # a one-GPU measurement: under torchrun the ranks skip it
    serving = None
    if args.serve_seconds > 0 and world == 1:
        serving = _section(serving_bench, args)
    _empty_cache()
    cpu = None
    parity = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(H, W)
        parity = _section(parity_vs_fp64_oracle, H, W)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    lat_sorted = sorted(lat)
    out = {
        "metric": METRIC, "value": round(value, 2), "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_max / args.steps, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f16",
        "data": "synthetic", "config": workload_config(H, W, world),
        "latency_ms": {"p50": round(float(np.percentile(lat_sorted, 50)), 3),
                       "p99": round(float(np.percentile(lat_sorted, 99)), 3)},
        "bytes_per_chunk": {"mean": int(np.mean(nbytes)), "min": int(min(nbytes)), "max": int(max(nbytes))},
        "enc_decomposed_fps": split,
        "precision_forms": forms,
        "batched": batched,
        "serving": serving,
        "reference_published": PUBLISHED,
        "intra": intra,
        "htl": htl,
        "ld": ld,
        "e2e": {"value": round(e2e, 2), "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "io": "8-bit YUV 4:2:0 planes in and out, converted on the device; copies on a second "
                      "stream, double-buffered, inside the timed region"},
        "gpu_launches": kernels_per_step * args.steps,
        "roofline": roof,
        "roofline_others": roof_others,
        "clocks": clk,
        "cpu_baseline": cpu,
        "parity": parity,
    }
    print(json.dumps(out), flush=True)


def main():
    args = parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
