"""Codec parity at the benchmarked configuration: 1920x1080 YUV 4:2:0 (padded to 1920x1088),
the benchmark's weights (calibrated seed-0 HT-S), QPs 0/21/42/63 one chunk after another, the GPU
codec through the drop-in proxies against the FP64 oracle (oracle/hts_oracle.py) run on the host
cores.  The assembled 1080p codec (arena layout, concatenation pitches, 32640-row phases, the
2.09 M-symbol compaction inside the phase graphs) is what these tests cover beyond the
small-size parity tests.

Tolerances (north-star targets, per chunk and so per QP): |PSNR_gpu - PSNR_oracle| <= 0.05 dB,
|bytes_gpu - bytes_oracle| <= 1 %; the fraction of quantised y latents that agree is reported
and must stay >= 97 % (HT-S) / 90 % (HT-L, LD; their random-init latents are larger, see
test_htl_gpu.py).  The encoder -> decoder round trip must be exact: entropy parameters, quantised
latents, y_hat and decoded features bit-identical between the two GPU instances.

Run with `-s` to see the per-QP table."""
import os
import sys

import numpy as np
import pytest
import torch

from dcvc_b200 import synthetic
from dcvc_b200.entropy_tables import add_cdf_to_state_dict
from dcvc_b200.model_spec import calibrated_hts_state_dict
from tests.hts_fixtures import make_proxy

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(__file__)), "oracle"))
import hts_oracle  # noqa: E402

pytestmark = pytest.mark.gpu

H, W = 1080, 1920
QPS = (0, 21, 42, 63)
THREADS = os.cpu_count() or 1


def _bench_state_dict():
    sd = add_cdf_to_state_dict(calibrated_hts_state_dict(0))
    return {k: (v.half().cuda() if v.is_floating_point() else v) for k, v in sd.items()}


def _psnr(frames_hat, frames):
    return float(np.mean([hts_oracle.psnr_yuv420(frames_hat[i].float().cpu(), *frames[i])[0]
                          for i in range(len(frames))]))


def test_hts_1080p_round_trip_exact():
    sd = _bench_state_dict()
    enc, dec = make_proxy(sd), make_proxy(sd)
    ref = synthetic.padded_reference_frame(synthetic.video_chunk_yuv420(2, H, W, 1, 0)[0])
    enc.add_ref_feature_from_frame(ref, True)
    dec.add_ref_feature_from_frame(ref, False)
    pr, pb = synthetic.padding_for(H, W)
    for k, (qp, reset) in enumerate([(0, False), (21, False), (42, True), (63, False)]):
        x = synthetic.to_model_input(synthetic.video_chunk_yuv420(2, H, W, 8, 8 * k))
        bits, ecp = enc.compress(x, qp, reset, pb, pr)
        out = dec.decompress(bits, qp, H, W, ecp, reset)
        torch.cuda.synchronize()
        assert len(out) == 8 and out[0].shape == (1, 3, H + pb, W + pr)
        for name in ("common", "y_q", "y_hat", "feature_p"):
            a, b = enc.buffer(name), dec.buffer(name)
            assert torch.equal(a.view(torch.int16), b.view(torch.int16)), (k, name)
        assert enc.stats()[0] == dec.stats()[0]


@pytest.fixture(scope="module")
def hts_oracle_chunks():
    """The FP64 oracle's run of the benchmark's 4 chunks (QPs 0/21/42/63 in order, one temporal
    state carried through): per chunk the source frames, payload size, mean PSNR and y_q.  Shared
    by every precision form."""
    sd16 = _bench_state_dict()
    sd_cpu = {k: v.cpu() for k, v in sd16.items()}
    oe = hts_oracle.HtsOracle(sd_cpu, 0.15, torch.float64, threads=THREADS)
    od = hts_oracle.HtsOracle(sd_cpu, 0.15, torch.float64)
    ref = synthetic.padded_reference_frame(synthetic.video_chunk_yuv420(2, H, W, 1, 0)[0], device="cpu")
    oe.add_ref_feature_from_frame(ref, True)
    od.add_ref_feature_from_frame(ref, False)
    pr, pb = synthetic.padding_for(H, W)
    out = []
    for k, qp in enumerate(QPS):
        frames = synthetic.video_chunk_yuv420(2, H, W, 8, 8 * k)
        x = synthetic.to_model_input(frames, device="cpu")
        r = oe.compress(x, qp, False, pb, pr)
        d = od.decompress(r["bit_stream"], qp, H, W, r["ec_parallel"], False)
        assert torch.equal(d["y_q"], r["y_q"])  # the oracle's own round trip is exact
        oq = r["y_q"][0].permute(1, 2, 0).reshape(-1, 256).float()
        out.append((qp, frames, r["bit_stream"].size, _psnr(d["x_hat"], frames), oq))
    return out


@pytest.mark.parametrize("precision", ["fp16", "bf16", "fp8"])
def test_hts_1080p_matches_fp64_oracle(precision, hts_oracle_chunks):
    from dcvc_b200.inference_extensions_cuda import DMCHTSProxy
    sd16 = _bench_state_dict()
    enc, dec = DMCHTSProxy(precision), DMCHTSProxy(precision)
    enc.set_param(sd16, 0.15)
    dec.set_param(sd16, 0.15)
    ref = synthetic.padded_reference_frame(synthetic.video_chunk_yuv420(2, H, W, 1, 0)[0])
    enc.add_ref_feature_from_frame(ref, True)
    dec.add_ref_feature_from_frame(ref, False)
    pr, pb = synthetic.padding_for(H, W)
    rows = []
    for k, (qp, frames, ob, po, oq) in enumerate(hts_oracle_chunks):
        # independent temporal state on each side, chunk after chunk as the benchmark runs them
        x = synthetic.to_model_input(frames)
        bits, ecp = enc.compress(x, qp, False, pb, pr)
        g = dec.decompress(bits, qp, H, W, ecp, False)
        torch.cuda.synchronize()
        for name in ("common", "y_q", "y_hat", "feature_p"):  # exact round trip in every form
            assert torch.equal(enc.buffer(name).view(torch.int16), dec.buffer(name).view(torch.int16))
        gq = enc.buffer("y_q").float().cpu()
        agree = float((gq == oq).float().mean())
        pg = _psnr(g, frames)
        rows.append((qp, pg, po, bits.size, ob, agree))
        print(f"HT-S {precision} 1080p qp {qp}: PSNR gpu {pg:.4f} oracle {po:.4f} "
              f"(d {pg - po:+.4f} dB), bytes gpu {bits.size} oracle {ob} "
              f"(d {100 * (bits.size - ob) / ob:+.3f} %), latents equal {100 * agree:.3f} %",
              flush=True)
    for qp, pg, po, gb, ob, agree in rows:
        assert abs(pg - po) <= 0.05, (precision, qp, pg, po)
        assert abs(gb - ob) <= 0.01 * ob, (precision, qp, gb, ob)
        assert agree >= 0.97, (precision, qp, agree)


def _restarted_parity(make, oracle_cls, sd16, ch_y, frames_per_call, qps, start_frames):
    """HT-L / LD form: every call starts both oracle instances from the GPU encoder's temporal
    memory (which the GPU decoder reproduces exactly), so the comparison is per call."""
    sd_cpu = {k: v.cpu() for k, v in sd16.items()}
    enc, dec = make(sd16), make(sd16)
    oe = oracle_cls(sd_cpu, 0.15, torch.float64)
    od = oracle_cls(sd_cpu, 0.15, torch.float64)
    torch.set_num_threads(THREADS)
    first = start_frames[0]
    ref = synthetic.padded_reference_frame(first)
    enc.add_ref_feature_from_frame(ref, True)
    dec.add_ref_feature_from_frame(ref, False)
    oe.add_ref_feature_from_frame(ref.cpu(), True)
    od.add_ref_feature_from_frame(ref.cpu(), False)
    pr, pb = synthetic.padding_for(H, W)
    H8, W8 = (H + pb) // 8, (W + pr) // 8
    rows = []
    for k, qp in enumerate(qps):
        if k > 0:
            memory = enc.buffer("memory").double().cpu().reshape(H8, W8, -1).permute(2, 0, 1)[None]
            oe.set_temporal_state(memory)
            od.set_temporal_state(memory)
        frames = start_frames[1 + k * frames_per_call: 1 + (k + 1) * frames_per_call]
        x = synthetic.to_model_input(frames)
        bits, ecp = enc.compress(x, qp, False, pb, pr)
        g = dec.decompress(bits, qp, H, W, ecp, False)
        g = g if isinstance(g, list) else [g]
        r = oe.compress(x.cpu(), qp, False, pb, pr)
        d = od.decompress(r["bit_stream"], qp, H, W, r["ec_parallel"], False)
        dx = d["x_hat"] if isinstance(d["x_hat"], list) else [d["x_hat"]]
        gq = enc.buffer("y_q").float().cpu()
        oq = r["y_q"][0].permute(1, 2, 0).reshape(-1, ch_y).float()
        agree = float((gq == oq).float().mean())
        pg, po = _psnr(g, frames), _psnr(dx, frames)
        rows.append((qp, pg, po, bits.size, r["bit_stream"].size, agree))
        assert torch.equal(d["y_q"], r["y_q"])
    return rows


def _check(name, rows, floor):
    for qp, pg, po, gb, ob, agree in rows:
        print(f"{name} 1080p qp {qp}: PSNR gpu {pg:.4f} oracle {po:.4f} (d {pg - po:+.4f} dB), "
              f"bytes gpu {gb} oracle {ob} (d {100 * (gb - ob) / ob:+.3f} %), "
              f"latents equal {100 * agree:.3f} %", flush=True)
    for qp, pg, po, gb, ob, agree in rows:
        assert abs(pg - po) <= 0.05, (name, qp, pg, po)
        assert abs(gb - ob) <= 0.01 * ob, (name, qp, gb, ob)
        assert agree >= floor, (name, qp, agree)


def test_htl_1080p_matches_fp64_oracle():
    import htl_oracle
    from tests.htl_fixtures import htl_state_dict16, make_htl_proxy
    frames = synthetic.video_chunk_yuv420(2, H, W, 1 + 8, 0)
    rows = _restarted_parity(make_htl_proxy, htl_oracle.HtlOracle, htl_state_dict16(), 256, 8,
                             (42,), frames)
    _check("HT-L", rows, 0.90)


def test_ld_1080p_matches_fp64_oracle():
    import ld_oracle
    from tests.ld_fixtures import ld_frames, ld_state_dict16, make_ld_proxy
    frames = ld_frames(H, W, 2)
    rows = _restarted_parity(make_ld_proxy, ld_oracle.LdOracle, ld_state_dict16(), ld_oracle.CH_Y,
                             1, (21, 42), frames)
    _check("LD", rows, 0.90)
