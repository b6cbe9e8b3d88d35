"""Intra (DMCI) model on CPU: the seeded weight spec, the oracle's sub-networks and the
multi-segment coder against the reference (golden fixtures from make_intra_golden.py), and
oracle round trips."""
import json
import os
import sys

import numpy as np
import pytest
import torch

from dcvc_b200 import MLCodec_extensions_cpp as M
from dcvc_b200.entropy_tables import add_cdf_to_state_dict
from dcvc_b200.model_spec import calibrated_dmci_state_dict, dmci_state_dict
from dcvc_b200 import synthetic

GOLD = os.path.join(os.path.dirname(__file__), "golden")
sys.path.insert(0, GOLD)
sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(__file__)), "oracle"))

from make_intra_golden import intra_module_inputs, segment_inputs  # noqa: E402
import hts_oracle  # noqa: E402
import intra_oracle  # noqa: E402


@pytest.fixture(scope="module")
def sd0():
    return dmci_state_dict(0)


def test_seed0_intra_weights_equal_reference(sd0):
    fp = json.load(open(os.path.join(GOLD, "weights_intra_seed0.json")))
    assert list(sd0.keys()) == list(fp.keys())
    for k, v in sd0.items():
        t = v.double().reshape(-1)
        f = fp[k]
        assert list(v.shape) == f["shape"], k
        assert [float(x) for x in t[:4]] == f["head"], k
        assert abs(float(t.sum()) - f["sum"]) <= 1e-9 * max(1.0, abs(f["sum"])), k
        assert abs(float((t * t).sum()) - f["sumsq"]) <= 1e-9 * max(1.0, f["sumsq"]), k
    assert sum(v.numel() for v in sd0.values()) == 42179328


def _close(a, ref):
    a = a.detach().float().numpy()
    scale = max(1.0, float(np.abs(ref).max()))
    assert a.shape == ref.shape
    err = float(np.abs(a - ref).max())
    assert err <= 1e-5 * scale, (err, scale)


def test_intra_modules_match_reference(sd0):
    o = intra_oracle.IntraOracle(add_cdf_to_state_dict(dict(sd0)), 0.15, torch.float64)
    g = np.load(os.path.join(GOLD, "intra_modules_golden.npz"))
    inp = intra_module_inputs()
    _close(o.encoder(inp["x"], inp["q_enc"]), g["encoder"])
    _close(o.hyper_encoder(torch.from_numpy(g["encoder"]).double()), g["hyper_encoder"])
    _close(o.hyper_decoder(inp["z_hat"]), g["hyper_decoder"])
    _close(o.prior_fusion(torch.from_numpy(g["hyper_decoder"]).double()), g["prior_fusion"])
    reduced = o.conv("y_spatial_prior_reduction.", inp["params"])
    _close(reduced, g["reduction"])
    for k in (1, 2, 3):
        _close(o.spatial_prior(k, inp["y_hat"], reduced), g[f"spatial_prior_{k}"])
    _close(o.decoder_features(inp["y_hat"], inp["q_dec"]), g["decoder"])


@pytest.fixture(scope="module")
def tables():
    g = np.load(os.path.join(GOLD, "cdf_tables.npz"))
    return [np.ascontiguousarray(g[k], np.int32) for k in ("qy", "ly", "qz", "lz")]


def test_segment_coders_match_reference_bytes(tables):
    qy, ly, qz, lz = tables
    g = np.load(os.path.join(GOLD, "rans_segments_golden.npz"))
    segs, z = segment_inputs()
    qp = int(g["qp"])
    assert g["counts"].tolist() == [s.size for s in segs]
    enc, dec = M.RansEncoder(), M.RansDecoder()
    for c in (enc, dec):
        c.set_cdf(qz, lz, 0)
        c.set_cdf(qy, ly, 1)
    ecps = sorted(int(k.split("_")[1]) for k in g.files if k.startswith("bytes_"))
    assert len(ecps) >= 4
    hts_oracle.use_reference_coder(False)
    for ecp in ecps:
        ref = g[f"bytes_{ecp}"]
        # C oracle
        b = hts_oracle.rans_encode_segments(qz, lz, qy, ly, segs, z, qp * 128, 128, ecp)
        assert b.tobytes() == ref.tobytes(), ecp
        # product coder, one encode_y per segment as the intra worker calls it
        enc.set_entropy_coder_parallel(ecp)
        enc.reset()
        for s in segs:
            enc.encode_y(s)
        enc.encode_z(z, qp * 128, 128)
        enc.flush()
        assert enc.get_encoded_stream().tobytes() == ref.tobytes(), ecp
        # incremental decoding, z first then the segments in reverse coding order
        dec.set_entropy_coder_parallel(ecp)
        dec.set_stream(ref)
        dec.decode_z(z.size, qp * 128, 128)
        assert (dec.get_decoded_tensor() == z).all()
        od = hts_oracle.RansSegmentDecoder(qz, lz, qy, ly, ref, ecp)
        assert (od.decode_z(z.size, qp * 128, 128) == z).all()
        for s in segs[::-1]:
            idx = (s.astype(np.int32) & 0xFF).astype(np.uint8)
            dec.decode_y(idx)
            want = (s.astype(np.int32) >> 8).astype(np.int8)
            assert (dec.get_decoded_tensor() == want).all(), ecp
            assert (od.decode_y(idx) == want).all(), ecp
        od.close()


@pytest.mark.parametrize("size,pad", [((64, 64), (0, 0)), ((56, 72), (8, 8))])
def test_intra_oracle_round_trip(size, pad):
    H, W = size
    sd = add_cdf_to_state_dict(calibrated_dmci_state_dict(0))
    o = intra_oracle.IntraOracle(sd, 0.15, torch.float64)
    y, u, v = synthetic.intra_frame_yuv420(1, H, W)
    x = synthetic.to_model_input([(y, u, v)], device="cpu")
    r = o.compress(x, 32, pad[0], pad[1])
    assert r["bit_stream"].size > 0 and len(r["symbols"]) == 4
    d = o.decompress(r["bit_stream"], 32, H, W, r["ec_parallel"])
    assert d["x_hat"].shape == (1, 3, H + pad[0], W + pad[1])
    assert torch.equal(d["y_q"], r["y_q"])
    assert float((d["y_hat"] - r["y_hat"]).abs().max()) < 1e-9
    assert float((d["x_hat"] - r["x_hat"]).abs().max()) < 1e-9
