"""The precision forms against the FP64 oracle at every QP (the precision-form configuration:
1920x1080 HT-S chunk, QPs 0..63, BF16 and FP8 forms beside the plain FP16 form).

Per QP, every form and the FP64 oracle (oracle/hts_oracle.py, host cores) start from the same
reference frame and code the same 8-frame chunk, so each QP is compared on its own.  Reported per
QP and form: PSNR-Y/U/V and the weighted (6Y+U+V)/8 PSNR deltas against the oracle, the payload
size delta in percent (bpp delta), the fraction of quantised latents equal to the oracle's, and
whether the decoder reproduced the encoder's entropy parameters, symbols and y_hat exactly.

Exactness is asserted for every form and QP.  The north-star error budget (|dPSNR| <= 0.05 dB,
|dbpp| <= 1 %) is asserted for the FP16 and BF16 forms; the FP8 form's deltas are reported
against the same budget (`within_budget` in the table) so that the QPs where E4M3 fits the
budget can be read off.

The oracle takes ~20 s per QP at 1080p, so the sweep runs only when DCVC_PRECISION_SWEEP=1;
DCVC_PRECISION_SWEEP_OUT=<path> also writes the table as JSON."""
import json
import os
import sys

import numpy as np
import pytest
import torch

from dcvc_b200 import synthetic
from dcvc_b200.entropy_tables import add_cdf_to_state_dict
from dcvc_b200.model_spec import calibrated_hts_state_dict

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(__file__)), "oracle"))
import hts_oracle  # noqa: E402

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(os.environ.get("DCVC_PRECISION_SWEEP") != "1",
                                 reason="set DCVC_PRECISION_SWEEP=1 to run the 64-QP sweep")]

H, W = 1080, 1920
FORMS = ("fp16", "bf16", "fp8")


def _psnr4(xs, frames):
    vals = np.array([hts_oracle.psnr_yuv420(xs[i].float().cpu(), *frames[i]) for i in range(len(frames))])
    return vals.mean(0)  # weighted, y, u, v


def test_precision_forms_at_every_qp():
    from dcvc_b200.inference_extensions_cuda import DMCHTSProxy
    torch.set_num_threads(os.cpu_count() or 1)
    sd = add_cdf_to_state_dict(calibrated_hts_state_dict(0))
    sd16 = {k: (v.half() if v.is_floating_point() else v) for k, v in sd.items()}
    sd_dev = {k: (v.cuda() if v.is_floating_point() else v) for k, v in sd16.items()}
    pr, pb = synthetic.padding_for(H, W)
    ref_planes = synthetic.video_chunk_yuv420(2, H, W, 1, 0)[0]
    frames = synthetic.video_chunk_yuv420(2, H, W, 8, 0)
    x_cpu = synthetic.to_model_input(frames, device="cpu")
    x_dev = x_cpu.cuda()
    ref_cpu = synthetic.padded_reference_frame(ref_planes, device="cpu")
    ref_dev = ref_cpu.cuda()
    proxies = {}
    for form in FORMS:
        enc, dec = DMCHTSProxy(form), DMCHTSProxy(form)
        enc.set_param(sd_dev, 0.15)
        dec.set_param(sd_dev, 0.15)
        proxies[form] = (enc, dec)
    table = []
    for qp in range(64):
        oe = hts_oracle.HtsOracle(sd16, 0.15, torch.float64)
        od = hts_oracle.HtsOracle(sd16, 0.15, torch.float64)
        oe.add_ref_feature_from_frame(ref_cpu, True)
        od.add_ref_feature_from_frame(ref_cpu, False)
        r = oe.compress(x_cpu, qp, False, pb, pr)
        d = od.decompress(r["bit_stream"], qp, H, W, r["ec_parallel"], False)
        po = _psnr4(d["x_hat"], frames)
        ob = r["bit_stream"].size
        oq = r["y_q"][0].permute(1, 2, 0).reshape(-1, 256).float()
        row = {"qp": qp, "oracle_bytes": int(ob), "oracle_psnr": round(float(po[0]), 4), "forms": {}}
        for form, (enc, dec) in proxies.items():
            enc.add_ref_feature_from_frame(ref_dev, True)
            dec.add_ref_feature_from_frame(ref_dev, False)
            bits, ecp = enc.compress(x_dev, qp, False, pb, pr)
            xs = dec.decompress(bits, qp, H, W, ecp, False)
            torch.cuda.synchronize()
            exact = all(torch.equal(enc.buffer(n).view(torch.int16), dec.buffer(n).view(torch.int16))
                        for n in ("common", "y_q", "y_hat"))
            pg = _psnr4(xs, frames)
            dp = pg - po
            dbpp = 100.0 * (bits.size - ob) / ob
            row["forms"][form] = {
                "dpsnr_db": round(float(dp[0]), 4), "dpsnr_y": round(float(dp[1]), 4),
                "dpsnr_u": round(float(dp[2]), 4), "dpsnr_v": round(float(dp[3]), 4),
                "dbpp_pct": round(dbpp, 3),
                "latent_agree": round(float((enc.buffer("y_q").float().cpu() == oq).float().mean()), 5),
                "round_trip_exact": exact,
                "within_budget": bool(abs(dp[0]) <= 0.05 and abs(dbpp) <= 1.0)}
        table.append(row)
        print(json.dumps(row), flush=True)
    out = os.environ.get("DCVC_PRECISION_SWEEP_OUT")
    if out:
        with open(out, "w") as f:
            json.dump(table, f)
    for row in table:
        for form in FORMS:
            assert row["forms"][form]["round_trip_exact"], (row["qp"], form)
        for form in ("fp16", "bf16"):
            f = row["forms"][form]
            assert abs(f["dpsnr_db"]) <= 0.05 and abs(f["dbpp_pct"]) <= 1.0, (row["qp"], form, f)
