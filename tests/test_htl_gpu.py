"""GPU HT-L chunk codec through the drop-in DMCHTLProxy: encoder and decoder state bit-identical
over chunks (reset and padded resolution included), corrupt-stream errors, and parity with the
FP64 oracle (oracle/htl_oracle.py) on the same seeded weights and inputs.

Parity tolerances (north-star targets, per chunk and so per QP): |PSNR_gpu - PSNR_oracle| <= 0.05
dB, |bytes_gpu - bytes_oracle| <= 1 %.  As a sanity floor beyond those, at least 90 % of the
quantised y latents equal: the random-init HT-L latents grow with the temporal memory (to ~100 by
the fourth chunk), where FP16 resolves 1/16 of a quantisation step, so a few per cent of them
round the other way than in FP64 (the HT-S model keeps 97 %)."""
import os
import sys

import numpy as np
import pytest
import torch

from dcvc_b200 import synthetic
from dcvc_b200._native import DcvcError
from tests.hts_fixtures import chunk, ref_frame
from tests.htl_fixtures import htl_state_dict16, make_htl_proxy

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(__file__)), "oracle"))
import hts_oracle  # noqa: E402
import htl_oracle  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("H,W", [(128, 192), (200, 248)])
def test_round_trip_exact(H, W):
    sd = htl_state_dict16()
    enc, dec = make_htl_proxy(sd), make_htl_proxy(sd)
    ref = ref_frame(H, W)
    enc.add_ref_feature_from_frame(ref, True)
    dec.add_ref_feature_from_frame(ref, False)
    pr, pb = synthetic.padding_for(H, W)
    for k, (qp, reset) in enumerate([(0, False), (21, False), (42, True), (63, False)]):
        bits, ecp = enc.compress(chunk(H, W, 8 * k), qp, reset, pb, pr)
        frames = dec.decompress(bits, qp, H, W, ecp, reset)
        torch.cuda.synchronize()
        assert len(frames) == 8 and frames[0].shape == (1, 3, H + pb, W + pr)
        # the decoder updates its temporal memory at the start of the next call, so the
        # entropy parameters, the latents and the decoded feature are what must agree here
        for name in ("common", "y_hat", "feature_p"):
            a, b = enc.buffer(name), dec.buffer(name)
            assert torch.equal(a.view(torch.int16), b.view(torch.int16)), (k, name)
        assert enc.stats()[0] == dec.stats()[0]
        assert all(float(f.abs().max()) <= 0.5 for f in frames)


def test_corrupt_stream_raises():
    sd = htl_state_dict16()
    enc, dec = make_htl_proxy(sd), make_htl_proxy(sd)
    H, W = 128, 128
    ref = ref_frame(H, W)
    enc.add_ref_feature_from_frame(ref, True)
    dec.add_ref_feature_from_frame(ref, False)
    bits, ecp = enc.compress(chunk(H, W, 0), 30, False, 0, 0)
    with pytest.raises(DcvcError):
        dec.decompress(bits[: max(1, bits.size // 5)], 30, H, W, ecp, False)


@pytest.mark.parametrize("H,W", [(128, 192), (200, 248)])
def test_gpu_matches_fp64_oracle(H, W):
    sd16 = htl_state_dict16()
    sd_cpu = {k: v.cpu() for k, v in sd16.items()}
    enc, dec = make_htl_proxy(sd16), make_htl_proxy(sd16)
    oe = htl_oracle.HtlOracle(sd_cpu, 0.15, torch.float64)
    od = htl_oracle.HtlOracle(sd_cpu, 0.15, torch.float64)
    ref = ref_frame(H, W)
    enc.add_ref_feature_from_frame(ref, True)
    dec.add_ref_feature_from_frame(ref, False)
    oe.add_ref_feature_from_frame(ref.cpu(), True)
    od.add_ref_feature_from_frame(ref.cpu(), False)
    pr, pb = synthetic.padding_for(H, W)
    H8, W8 = (H + pb) // 8, (W + pr) // 8

    def state(proxy, name):
        t = proxy.buffer(name).double().cpu()
        return t.reshape(H8, W8, -1).permute(2, 0, 1)[None]

    for k, qp in enumerate([0, 21, 42, 63]):
        if k > 0:
            # The random-init HT-L recurrence amplifies rounding differences from chunk to chunk
            # (its temporal memory grows about 2x per chunk), so every chunk starts both oracle
            # instances from the GPU encoder's temporal memory (which the GPU decoder reproduces
            # exactly): the comparison is per chunk, i.e. per QP.
            memory = state(enc, "memory")
            oe.set_temporal_state(memory)
            od.set_temporal_state(memory)
        frames = synthetic.video_chunk_yuv420(2, H, W, 8, 8 * k)
        x = synthetic.to_model_input(frames)
        bits, ecp = enc.compress(x, qp, False, pb, pr)
        g = dec.decompress(bits, qp, H, W, ecp, False)
        r = oe.compress(x.cpu(), qp, False, pb, pr)
        d = od.decompress(r["bit_stream"], qp, H, W, r["ec_parallel"], False)
        gq = enc.buffer("y_q").float().cpu()
        oq = r["y_q"][0].permute(1, 2, 0).reshape(-1, 256).float()
        agree = float((gq == oq).float().mean())
        pg = np.mean([hts_oracle.psnr_yuv420(g[i].float(), *frames[i])[0] for i in range(8)])
        po = np.mean([hts_oracle.psnr_yuv420(d["x_hat"][i], *frames[i])[0] for i in range(8)])
        assert abs(pg - po) <= 0.05, (k, pg, po)
        ob = r["bit_stream"].size
        assert abs(bits.size - ob) <= 0.01 * ob, (k, bits.size, ob)
        assert agree >= 0.90, (k, agree)
        assert torch.equal(d["y_q"], r["y_q"])
