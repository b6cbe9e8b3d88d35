"""Low-delay (LD) model on CPU: the seeded weight spec and the oracle's sub-networks against the
reference (golden fixtures from make_ld_golden.py), and oracle round trips over frames with a
reset."""
import json
import os
import sys

import numpy as np
import pytest
import torch

from dcvc_b200 import synthetic
from dcvc_b200.entropy_tables import add_cdf_to_state_dict
from dcvc_b200.model_spec import calibrated_ld_state_dict, ld_state_dict

GOLD = os.path.join(os.path.dirname(__file__), "golden")
sys.path.insert(0, GOLD)
sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(__file__)), "oracle"))

from make_ld_golden import ld_module_inputs  # noqa: E402
import ld_oracle  # noqa: E402


@pytest.fixture(scope="module")
def sd0():
    return ld_state_dict(0)


def test_seed0_ld_weights_equal_reference(sd0):
    fp = json.load(open(os.path.join(GOLD, "weights_ld_seed0.json")))
    assert list(sd0.keys()) == list(fp.keys())
    for k, v in sd0.items():
        t = v.double().reshape(-1)
        f = fp[k]
        assert list(v.shape) == f["shape"], k
        assert [float(x) for x in t[:4]] == f["head"], k
        assert abs(float(t.sum()) - f["sum"]) <= 1e-9 * max(1.0, abs(f["sum"])), k
        assert abs(float((t * t).sum()) - f["sumsq"]) <= 1e-9 * max(1.0, f["sumsq"]), k
    assert sum(v.numel() for v in sd0.values()) == 9650176


def _close(a, ref):
    a = a.detach().float().numpy()
    scale = max(1.0, float(np.abs(ref).max()))
    assert a.shape == ref.shape
    err = float(np.abs(a - ref).max())
    assert err <= 1e-5 * scale, (err, scale)


def test_ld_modules_match_reference(sd0):
    o = ld_oracle.LdOracle(add_cdf_to_state_dict(dict(sd0)), 0.15, torch.float64)
    g = np.load(os.path.join(GOLD, "ld_modules_golden.npz"))
    inp = ld_module_inputs()
    _close(o.encoder(inp["x"], inp["ctx"], inp["q_enc"]), g["encoder"])
    _close(o.hyper_encoder(torch.from_numpy(g["encoder"]).double()), g["hyper_encoder"])
    _close(o.hyper_decoder(inp["z_hat"]), g["hyper_decoder"])
    _close(o.temporal_prior_ld(inp["memory"]), g["temporal_prior_encoder"])
    _close(o.prior_fusion_ld(torch.from_numpy(g["hyper_decoder"]).double(),
                             torch.from_numpy(g["temporal_prior_encoder"]).double(), inp["q_feat"]),
           g["prior_fusion"])
    _close(o.spatial_prior_ld(inp["y_hat"], inp["params"]), g["spatial_prior"])
    _close(o.decoder(inp["y_hat"], inp["ctx"], inp["q_dec"]), g["decoder"])
    head = o.recon_head_out(inp["feature"])
    _close(head, g["recon_reset"])
    _close(torch.nn.functional.pixel_shuffle(head, 8), g["recon"])
    _close(o.feature_adaptor_i(inp["feature_i"]), g["feature_adaptor_i"])
    _close(o.feature_adaptor_m(inp["memory"], inp["feature"]), g["feature_adaptor_m"])
    _close(o.feature_extractor(inp["memory"]), g["feature_extractor"])


def test_ld_oracle_round_trip():
    H, W = 48, 64
    sd = add_cdf_to_state_dict(calibrated_ld_state_dict(0))
    oe = ld_oracle.LdOracle(sd, 0.15, torch.float64)
    od = ld_oracle.LdOracle(sd, 0.15, torch.float64)
    frames = synthetic.video_chunk_yuv420(2, H, W, 5, 0)
    ref = synthetic.padded_reference_frame(frames[0], device="cpu")
    oe.add_ref_feature_from_frame(ref, True)
    od.add_ref_feature_from_frame(ref, False)
    pr, pb = synthetic.padding_for(H, W)
    for k, (qp, reset) in enumerate([(21, False), (42, True), (0, False), (63, False)]):
        x = synthetic.to_model_input([frames[k + 1]], device="cpu")
        r = oe.compress(x, qp, reset, pb, pr)
        d = od.decompress(r["bit_stream"], qp, H, W, r["ec_parallel"], reset)
        assert torch.equal(d["y_q"], r["y_q"]), k
        assert float((d["y_hat"] - r["y_hat"]).abs().max()) < 1e-9, k
        assert d["x_hat"].shape == (1, 3, H + pb, W + pr)
