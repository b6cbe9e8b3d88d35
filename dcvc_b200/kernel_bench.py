"""Micro-benchmark of the codec's kernels at their 1080p shapes (CUDA events on the launching
stream), also the small fixed case used for ncu captures.

    python -m dcvc_b200.kernel_bench [--case quad|quad_f8|wsilu|res|dwres|dwres_split|bias2048|dwconv|ffn|ffn_ld|unshuffle|shuffle|quantize|rans|all]
                                     [--reps N] [--sets S] [--bn 0|64|128|256|-1]

(--bn -1 selects the streaming form of the residual GEMM.)

Consecutive launches cycle through S independent operand sets (default: enough sets for 300 MB),
so the timed launches read their inputs from HBM rather than from the 126 MB L2, as they do
inside a chunk.

Shapes are those of a 512-channel dcb2 DepthConvBlock at 1920x1088 (M = 136 x 240 = 32640
pixels): dc.0 (512 -> 256, WSiLU), depthwise 3x3 on 256 channels, dc.3 (256 -> 512 + residual),
ffn.0 (512 -> 4 x 256, WSiLU chunk-add), and the encoder's 2048 -> 512 adaptor.  `dwres` is the
depthwise 3x3 and dc.3 in one launch (the depthwise form of the streaming residual GEMM),
`dwres_split` the same two steps as two launches.
"""
import argparse
import json

import torch

from . import _native as N
from . import ops

M8 = 136 * 240


def _case(name, g, bn=0):
    def rnd(*s, scale=1.0):
        return (torch.randn(*s, device="cuda", generator=g) * scale).half()

    if name in ("ffn", "ffn_ld"):
        # the fused ConvFFN (quad GEMM + residual GEMM in one kernel) of a 512-channel dcb2 block
        # ("ffn") or of a 256-channel one, the LD codec's ("ffn_ld")
        C = 512 if name == "ffn" else 256
        cf = C // 2
        x = rnd(M8, C)
        w1, w2 = rnd(4 * cf, C, scale=C ** -0.5), rnd(C, cf, scale=cf ** -0.5)
        b1 = torch.zeros(4 * cf, device="cuda")
        b2 = torch.zeros(C, device="cuda")
        out = torch.empty_like(x)
        fn = lambda: ops.conv_ffn(x, w1, b1, w2, b2, out=out, block_n=bn)  # noqa: E731
        return fn, 2.0 * M8 * (4 * cf * C + C * cf), (2 * x.numel() + w1.numel() + w2.numel()) * 2
    if name == "quad_f8":
        # ffn.0 of a 512-channel block in the FP8 form: E4M3 operands, per-row scales, BF16 out
        a = rnd(M8, 512).to(torch.float8_e4m3fn)
        w = rnd(1024, 512, scale=512 ** -0.5)
        ws = (w.float().abs().amax(1) / 448.0).contiguous()
        wq = (w.float() / ws[:, None]).to(torch.float8_e4m3fn)
        b = torch.zeros(1024, device="cuda")
        out = torch.empty(M8, 256, device="cuda", dtype=torch.bfloat16)
        fn = lambda: ops.conv1x1_f8(a, wq, ws, b, N.EPI_QUAD, out=out, block_n=bn)  # noqa: E731
        return fn, 2.0 * M8 * 1024 * 512, (M8 * 512 + 1024 * 512) + M8 * 256 * 2
    if name == "unshuffle":
        # pad_and_unshuffle_8 of one 1080p input chunk: [1080, 1920, 24] -> [136 x 240, 1536]
        x = rnd(1080, 1920, 24)
        out = torch.empty(M8, 1536, device="cuda", dtype=torch.float16)
        fn = lambda: ops.pad_unshuffle8(x, 8, 0, out=out)  # noqa: E731
        return fn, 0.0, (x.numel() + out.numel()) * 2
    if name == "shuffle":
        # pixel_shuffle(8) + clamp of one reconstructed 1080p frame: [136 x 240, 192] -> [1088, 1920, 3]
        x = rnd(M8, 192)
        out = torch.empty(1088, 1920, 3, device="cuda", dtype=torch.float16)

        def fn():
            N.check(N.lib.dcvc_shuffle8_clamp(x.data_ptr(), 136, 240, 3, 192, out.data_ptr(),
                                              torch.cuda.current_stream().cuda_stream), "shuffle8_clamp")
        return fn, 0.0, (x.numel() + out.numel()) * 2
    if name == "quantize":
        # the last masked quantisation phase at 1080p (y: 68 x 120 x 256, mode 2: accumulate and
        # scale by max(q_dec, 0.5)); reads y, scales, means, q_dec, y_q, y_hat, writes y_q, y_hat
        M16 = 68 * 120
        y, sc, mu, qd = rnd(M16, 256), rnd(M16, 256).abs(), rnd(M16, 256), rnd(M16, 256).abs()
        yq, yh = torch.zeros_like(y), torch.zeros_like(y)
        fn = lambda: ops.quantize_phase(3, 2, y, sc, mu, qd, 0.15, yq, yh, 68, 120)  # noqa: E731
        return fn, 0.0, 8 * y.numel() * 2
    if name in ("dwres", "dwres_split"):
        # depthwise 3x3 on dc.0's 256-channel output, then dc.3 (256 -> 512) + bias + residual
        x = rnd(M8, 256)
        dw = torch.randn(9, 256, device="cuda", generator=g)
        w = rnd(512, 256, scale=256 ** -0.5)
        b = torch.zeros(512, device="cuda")
        res = rnd(M8, 512)
        out = torch.empty(M8, 512, device="cuda", dtype=torch.float16)
        if name == "dwres":
            fn = lambda: ops.dw3x3_conv1x1_res(x, 136, 240, dw, w, b, res, out=out)  # noqa: E731
        else:
            t = torch.empty_like(x)

            def fn():
                ops.dwconv3x3(x, 136, 240, dw, t)
                ops.conv1x1(t, w, b, N.EPI_BIAS_RES, res=res, out=out, block_n=N.BLOCK_N_STREAM)
        return fn, 2.0 * M8 * 512 * 256, (x.numel() + w.numel() + 2 * res.numel()) * 2 + dw.numel() * 4
    if name == "dwconv":
        x = rnd(M8, 256)
        w = torch.randn(9, 256, device="cuda", generator=g)
        out = torch.empty_like(x)
        fn = lambda: ops.dwconv3x3(x, 136, 240, w, out)  # noqa: E731
        return fn, 0.0, 2 * x.numel() * 2 + w.numel() * 4
    shapes = {"quad": (M8, 1024, 512, N.EPI_QUAD), "wsilu": (M8, 256, 512, N.EPI_BIAS_WSILU),
              "res": (M8, 512, 256, N.EPI_BIAS_RES), "bias2048": (M8, 512, 2048, N.EPI_BIAS),
              # launch and ramp cost: one tile, and the residual GEMM at a quarter of the pixels
              "tiny": (128, 256, 64, N.EPI_BIAS), "res_quarter": (M8 // 4, 512, 256, N.EPI_BIAS_RES),
              # the y-level (M / 4) dc.0 and quad GEMMs of a 512-channel block
              "wsilu_quarter": (M8 // 4, 256, 512, N.EPI_BIAS_WSILU),
              "quad_quarter": (M8 // 4, 1024, 512, N.EPI_QUAD),
              # the recon head's 256-channel blocks (8 frames x 3 per decoded chunk) and the
              # y-level residual GEMMs at K = 512
              "wsilu256": (M8, 256, 256, N.EPI_BIAS_WSILU), "res256": (M8, 256, 256, N.EPI_BIAS_RES),
              "quad256": (M8, 1024, 256, N.EPI_QUAD), "res512y": (M8 // 4, 512, 512, N.EPI_BIAS_RES)}
    M, Nn, K, epi = shapes[name]
    a = rnd(M, K)
    w = rnd(Nn, K, scale=K ** -0.5)
    b = torch.zeros(Nn, device="cuda")
    res = rnd(M, Nn) if epi == N.EPI_BIAS_RES else None
    nout = Nn // 4 if epi == N.EPI_QUAD else Nn
    out = torch.empty(M, nout, device="cuda", dtype=torch.float16)
    fn = lambda: ops.conv1x1(a, w, b, epi, res=res, out=out, block_n=bn)  # noqa: E731
    byts = (M * K + Nn * K + M * nout + (M * Nn if res is not None else 0)) * 2
    return fn, 2.0 * M * Nn * K, byts


def run(name, reps=20, warmup=5, sets=0, bn=0):
    """Device time per launch: `reps` launches cycling through the operand sets are captured in
    one CUDA graph (no host launch cost between them, as inside the codec's phase graphs), the
    graph is replayed once to warm up and timed on the next replay."""
    g = torch.Generator(device="cuda").manual_seed(11)
    made = [_case(name, g, bn)]
    if sets <= 0:
        sets = -(-300_000_000 // made[0][2])
    made += [_case(name, g, bn) for _ in range(sets - 1)]
    fns = [m[0] for m in made]
    flops, byts = made[0][1], made[0][2]
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        for i in range(warmup):
            fns[i % len(fns)]()
        stream.synchronize()
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph, stream=stream):
            for i in range(reps):
                fns[i % len(fns)]()
        graph.replay()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(stream)
        graph.replay()
        e.record(stream)
    e.synchronize()
    sec = s.elapsed_time(e) / 1e3 / reps
    return {"case": name, "bn": bn, "us": round(sec * 1e6, 2), "tflops": round(flops / sec / 1e12, 1),
            "gbs": round(byts / sec / 1e9, 1)}


def rans(reps=5):
    """rANS coding of one 1080p payload (y symbols of an HT-S chunk at a mid rate plus its z) on
    the GPU (one warp per payload, one thread per sub-stream) and on the host threads, and of a
    batch of 32 such payloads (independent streams) in one GPU launch.  Same bytes either way."""
    import time

    import numpy as np

    from . import MLCodec_extensions_cpp as M
    from .entropy_tables import gaussian_tables
    from .rans_gpu import GpuRansCoder
    qy, ly = gaussian_tables()
    qz = np.tile(qy[:1], (64 * 128, 1)).astype(np.int32)
    lz = np.tile(ly[:1], 64 * 128).astype(np.int32)
    rng = np.random.default_rng(3)
    ny, nz = 300000, 128 * 17 * 30
    q = np.clip(np.round(rng.laplace(0, 1.2, ny)), -128, 127).astype(np.int64)
    y = ((q << 8) + rng.integers(8, 40, ny)).astype(np.int16)
    z = np.clip(np.round(rng.laplace(0, 1.0, nz)), -64, 63).astype(np.int8)
    ecp = M.ec_parallel_for(ny)
    g = GpuRansCoder(qz, lz, qy, ly)
    yd, zd = torch.from_numpy(y).cuda(), torch.from_numpy(z).cuda()
    job = {"y": yd, "z": zd, "z_offset": 0, "z_ch": 128, "ecp": ecp}
    out = {"case": "rans", "symbols": ny + nz, "ec_parallel": ecp}
    for name, jobs in (("gpu_1", [job]), ("gpu_32", [job] * 32)):
        g.encode(jobs)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(reps):
            outs, st = g.encode(jobs)
        torch.cuda.synchronize()
        te = (time.perf_counter() - t0) / reps
        djobs = [{"data": outs[0], "ecp": ecp, "n_z": nz, "z_offset": 0, "z_ch": 128,
                  "y_idx": (yd & 0xff).to(torch.uint8)}] * len(jobs)
        g.decode(djobs)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(reps):
            g.decode(djobs)
        torch.cuda.synchronize()
        td = (time.perf_counter() - t0) / reps
        out[name] = {"payloads": len(jobs), "enc_ms": round(te * 1e3, 3), "dec_ms": round(td * 1e3, 3)}
    enc = M.RansEncoder()
    enc.set_cdf(qz, lz, 0)
    enc.set_cdf(qy, ly, 1)
    enc.set_entropy_coder_parallel(ecp)
    t0 = time.perf_counter()
    for _ in range(reps):
        enc.reset()
        enc.encode_y(y)
        enc.encode_z(z, 0, 128)
        enc.flush()
    te = (time.perf_counter() - t0) / reps
    ref = enc.get_encoded_stream()
    dec = M.RansDecoder()
    dec.set_cdf(qz, lz, 0)
    dec.set_cdf(qy, ly, 1)
    dec.set_entropy_coder_parallel(ecp)
    idx = (y & 0xff).astype(np.uint8)
    t0 = time.perf_counter()
    for _ in range(reps):
        dec.set_stream(ref)
        dec.decode_z(nz, 0, 128)
        dec.decode_y(idx)
    td = (time.perf_counter() - t0) / reps
    out["cpu_1"] = {"payloads": 1, "enc_ms": round(te * 1e3, 3), "dec_ms": round(td * 1e3, 3)}
    out["bytes"] = int(ref.size)
    out["identical"] = bool(outs[0].cpu().numpy().tobytes() == ref.tobytes())
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--case", default="all")
    ap.add_argument("--reps", type=int, default=20)
    ap.add_argument("--sets", type=int, default=0)
    ap.add_argument("--bn", type=int, default=0,
                    help="GEMM N tile (0 = the library's choice, -1 = streaming residual form)")
    args = ap.parse_args()
    cases = ["quad", "wsilu", "res", "bias2048", "dwconv", "ffn"] if args.case == "all" else [args.case]
    for c in cases:
        if c == "rans":
            print(json.dumps(rans()), flush=True)
            continue
        print(json.dumps(run(c, args.reps, sets=args.sets, bn=args.bn)), flush=True)


if __name__ == "__main__":
    main()
