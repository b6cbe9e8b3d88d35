"""Pins the network oracle (oracle/hts_oracle.py) against the reference nn.Modules: outputs of
every HT-S sub-network for seeded inputs (tests/golden/modules_golden.npz, generated from the
reference by tests/golden/make_golden.py) in float64."""
import os
import sys

import numpy as np
import pytest
import torch

from dcvc_b200.model_spec import hts_state_dict

GOLD = os.path.join(os.path.dirname(__file__), "golden")
sys.path.insert(0, GOLD)
sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(__file__)), "oracle"))

from make_modules_golden import module_inputs  # noqa: E402
import hts_oracle  # noqa: E402


@pytest.fixture(scope="module")
def oracle():
    sd = hts_state_dict(0)
    from dcvc_b200.entropy_tables import add_cdf_to_state_dict
    return hts_oracle.HtsOracle(add_cdf_to_state_dict(sd), 0.15, torch.float64)


@pytest.fixture(scope="module")
def gold():
    return np.load(os.path.join(GOLD, "modules_golden.npz"))


def _close(a, ref):
    a = a.detach().float().numpy()
    scale = max(1.0, float(np.abs(ref).max()))
    assert a.shape == ref.shape
    err = float(np.abs(a - ref).max())
    assert err <= 1e-5 * scale, (err, scale)


def test_modules_match_reference(oracle, gold):
    o = oracle
    inp = module_inputs()
    y = o.encoder(inp["x"], inp["ctx"], inp["q_enc"])
    _close(y, gold["encoder"])
    _close(o.hyper_encoder(torch.from_numpy(gold["encoder"]).double()), gold["hyper_encoder"])
    _close(o.hyper_decoder(inp["z_hat"]), gold["hyper_decoder"])
    tp = o.temporal_prior(inp["memory"], inp["q_feat"])
    _close(tp, gold["temporal_prior_encoder"])
    pf = o.prior_fusion(torch.from_numpy(gold["hyper_decoder"]).double(),
                        torch.from_numpy(gold["temporal_prior_encoder"]).double())
    _close(pf, gold["prior_fusion"])
    reduced = o.conv("y_spatial_prior_reduction.", inp["params"])
    _close(reduced, gold["reduction"])
    for k in (1, 2, 3):
        _close(o.spatial_prior(k, inp["y_hat"], reduced), gold[f"spatial_prior_{k}"])
    _close(o.decoder(inp["y_hat"], inp["ctx"], inp["q_dec"]), gold["decoder"])
    frames = []
    for i in range(8):
        if i % 2 == 0:
            common = o.dcb(f"recon_head.conv1.{i // 2}.0.", inp["feature"])
        frames.append(torch.nn.functional.pixel_shuffle(o.recon_head_frame(i, common), 8))
    for i in range(8):
        _close(frames[i], gold[f"recon_{i}"])
    _close(o.recon_head_reset(inp["feature"]), gold["recon_reset"])
    _close(o.feature_adaptor_i(inp["feature_i"]), gold["feature_adaptor_i"])
    _close(o.feature_adaptor_m(inp["memory"], inp["feature"]), gold["feature_adaptor_m"])
    _close(o.feature_extractor(inp["memory"]), gold["feature_extractor"])


def test_scale_index_table_matches_product():
    """The oracle's NumPy restatement of the scale->index table equals the product's C++ table
    (read back through the mask/quant kernels' host builder)."""
    import ctypes
    from dcvc_b200 import _native as N
    N.lib.dcvc_scale_index_table.restype = ctypes.c_int
    N.lib.dcvc_scale_index_table.argtypes = [ctypes.c_void_p]
    prod = np.zeros(65536, np.uint8)
    assert N.lib.dcvc_scale_index_table(prod.ctypes.data) == 0
    assert (hts_oracle.scale_index_lut() == prod).all()
    # spot values: the minimum scale maps to table 0, the maximum to table 127
    assert hts_oracle.scale_index([0.11, 16.0, 1000.0, -3.0]).tolist() == [0, 127, 127, 0]
