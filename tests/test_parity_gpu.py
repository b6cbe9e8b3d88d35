"""GPU HT-S codec against the FP64 oracle (oracle/hts_oracle.py) on the same seeded weights and
inputs, chunk by chunk with independent temporal state on each side.

Tolerances (north-star targets): |PSNR_gpu - PSNR_oracle| <= 0.05 dB and
|bpp_gpu - bpp_oracle| <= 1 % per chunk; at least 97 % of the quantised y latents equal (the
FP16 GPU state and the FP64 oracle state drift apart slowly over chunks)."""
import os
import sys

import numpy as np
import pytest
import torch

from dcvc_b200 import synthetic
from tests.hts_fixtures import make_proxy, state_dict

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(__file__)), "oracle"))
import hts_oracle  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("H,W", [(128, 192), (200, 248)])
def test_gpu_matches_fp64_oracle(H, W):
    sd16 = state_dict()
    sd_cpu = {k: v.cpu() for k, v in sd16.items()}
    enc, dec = make_proxy(sd16), make_proxy(sd16)
    oe = hts_oracle.HtsOracle(sd_cpu, 0.15, torch.float64)
    od = hts_oracle.HtsOracle(sd_cpu, 0.15, torch.float64)
    ref = synthetic.padded_reference_frame(synthetic.video_chunk_yuv420(2, H, W, 1, 0)[0])
    enc.add_ref_feature_from_frame(ref, True)
    dec.add_ref_feature_from_frame(ref, False)
    oe.add_ref_feature_from_frame(ref.cpu(), True)
    od.add_ref_feature_from_frame(ref.cpu(), False)
    pr, pb = synthetic.padding_for(H, W)
    for k, qp in enumerate([0, 21, 42, 63]):
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
        assert abs(bits.size - r["bit_stream"].size) <= 0.01 * r["bit_stream"].size, (k, bits.size, r["bit_stream"].size)
        assert agree >= 0.97, (k, agree)
        # the oracle's own round trip is exact
        assert torch.equal(d["y_q"], r["y_q"])
