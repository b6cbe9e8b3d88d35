"""GPU low-delay (LD) frame codec through the drop-in DMCLDProxy: encoder and decoder state
bit-identical over frames (reset and padded resolution included), corrupt-stream errors, and
parity with the FP64 oracle (oracle/ld_oracle.py) on the same seeded weights and inputs.

Parity tolerances (the HT-S targets, per frame): |PSNR_gpu - PSNR_oracle| <= 0.05 dB and
|bytes_gpu - bytes_oracle| <= 1 %, with at least 90 % of the quantised y latents equal as a
sanity floor (FP16 against FP64 rounds a few latents near a half-step the other way)."""
import os
import sys

import pytest
import torch

from dcvc_b200 import synthetic
from dcvc_b200._native import DcvcError
from tests.ld_fixtures import ld_frames, ld_state_dict16, make_ld_proxy

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(__file__)), "oracle"))
import hts_oracle  # noqa: E402
import ld_oracle  # noqa: E402

pytestmark = pytest.mark.gpu


def _pair(sd, frames):
    enc, dec = make_ld_proxy(sd), make_ld_proxy(sd)
    ref = synthetic.padded_reference_frame(frames[0])
    enc.add_ref_feature_from_frame(ref, True)
    dec.add_ref_feature_from_frame(ref, False)
    return enc, dec


@pytest.mark.parametrize("H,W", [(128, 192), (200, 248)])
def test_round_trip_exact(H, W):
    sd = ld_state_dict16()
    frames = ld_frames(H, W, 5)
    enc, dec = _pair(sd, frames)
    pr, pb = synthetic.padding_for(H, W)
    for k, (qp, reset) in enumerate([(0, False), (21, False), (42, True), (63, False),
                                     (30, False)]):
        x = synthetic.to_model_input([frames[k + 1]])
        bits, ecp = enc.compress(x, qp, reset, pb, pr)
        x_hat = dec.decompress(bits, qp, H, W, ecp, reset)
        torch.cuda.synchronize()
        assert x_hat.shape == (1, 3, H + pb, W + pr)
        # the decoder updates its temporal memory at the start of the next call, so the
        # entropy parameters, the latents and the decoded feature are what must agree here
        for name in ("common", "y_hat", "feature_p"):
            a, b = enc.buffer(name), dec.buffer(name)
            assert torch.equal(a.view(torch.int16), b.view(torch.int16)), (k, name)
        assert enc.stats()[0] == dec.stats()[0]
        assert float(x_hat.abs().max()) <= 0.5


def test_corrupt_stream_raises():
    sd = ld_state_dict16()
    H, W = 128, 128
    frames = ld_frames(H, W, 1)
    enc, dec = _pair(sd, frames)
    bits, ecp = enc.compress(synthetic.to_model_input([frames[1]]), 30, False, 0, 0)
    with pytest.raises(DcvcError):
        dec.decompress(bits[: max(1, bits.size // 5)], 30, H, W, ecp, False)


def test_bad_arguments_raise():
    sd = ld_state_dict16()
    H, W = 64, 64
    frames = ld_frames(H, W, 1)
    enc, _ = _pair(sd, frames)
    x = synthetic.to_model_input([frames[1]])
    with pytest.raises(DcvcError):
        enc.compress(x, 64, False, 0, 0)            # qp out of range
    with pytest.raises(DcvcError):
        enc.compress(x[:, :, :48], 0, False, 0, 0)  # size differs from the reference frame
    with pytest.raises(ValueError):
        enc.compress(synthetic.to_model_input(frames[:2]), 0, False, 0, 0)


@pytest.mark.parametrize("H,W", [(128, 192), (200, 248)])
def test_gpu_matches_fp64_oracle(H, W):
    sd16 = ld_state_dict16()
    sd_cpu = {k: v.cpu() for k, v in sd16.items()}
    frames = ld_frames(H, W, 4)
    enc, dec = _pair(sd16, frames)
    oe = ld_oracle.LdOracle(sd_cpu, 0.15, torch.float64)
    od = ld_oracle.LdOracle(sd_cpu, 0.15, torch.float64)
    ref = synthetic.padded_reference_frame(frames[0], device="cpu")
    oe.add_ref_feature_from_frame(ref, True)
    od.add_ref_feature_from_frame(ref, False)
    pr, pb = synthetic.padding_for(H, W)
    H8, W8 = (H + pb) // 8, (W + pr) // 8

    def state(proxy, name):
        t = proxy.buffer(name).double().cpu()
        return t.reshape(H8, W8, -1).permute(2, 0, 1)[None]

    for k, qp in enumerate([0, 21, 42, 63]):
        if k > 0:
            # Every frame starts both oracle instances from the GPU encoder's temporal memory
            # (which the GPU decoder reproduces exactly), so that rounding differences do not
            # accumulate through the random-init recurrence: the comparison is per frame.
            memory = state(enc, "memory")
            oe.set_temporal_state(memory)
            od.set_temporal_state(memory)
        x = synthetic.to_model_input([frames[k + 1]])
        bits, ecp = enc.compress(x, qp, False, pb, pr)
        g = dec.decompress(bits, qp, H, W, ecp, False)
        r = oe.compress(x.cpu(), qp, False, pb, pr)
        d = od.decompress(r["bit_stream"], qp, H, W, r["ec_parallel"], False)
        gq = enc.buffer("y_q").float().cpu()
        oq = r["y_q"][0].permute(1, 2, 0).reshape(-1, ld_oracle.CH_Y).float()
        agree = float((gq == oq).float().mean())
        pg = hts_oracle.psnr_yuv420(g.float(), *frames[k + 1])[0]
        po = hts_oracle.psnr_yuv420(d["x_hat"], *frames[k + 1])[0]
        assert abs(pg - po) <= 0.05, (k, pg, po)
        ob = r["bit_stream"].size
        assert abs(bits.size - ob) <= 0.01 * ob, (k, bits.size, ob)
        assert agree >= 0.90, (k, agree)
        assert torch.equal(d["y_q"], r["y_q"])
