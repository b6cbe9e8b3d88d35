"""Reference nn.Module outputs for small seeded inputs (float64), used to pin the network oracle.

Called by make_golden.py with the seed-0 reference HT-S model.  Inputs are regenerated on the
test side from the same seeds (torch CPU generator), so only the outputs are stored.
"""
import os

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))

# 128 x 64 frames: H8 x W8 = 16 x 8, y level 8 x 4, z level 2 x 1
H, W = 128, 64


def module_inputs():
    g = torch.Generator().manual_seed(2024)
    r = lambda *s: torch.rand(*s, generator=g, dtype=torch.float64)  # noqa: E731
    h8, w8 = H // 8, W // 8
    return {
        "x": r(1, 24, H, W) - 0.5,
        "ctx": r(1, 512, h8, w8) * 2 - 1,
        "memory": r(1, 512, h8, w8) * 2 - 1,
        "feature": r(1, 512, h8, w8) * 2 - 1,
        "feature_i": r(1, 192, h8, w8) - 0.5,
        "q_enc": r(1, 512, 1, 1) + 0.5,
        "q_dec": r(1, 512, 1, 1) + 0.5,
        "q_feat": r(1, 512, 1, 1) + 0.5,
        "z_hat": torch.round((r(1, 128, h8 // 8, w8 // 8) - 0.5) * 8),
        "y_hat": (r(1, 256, h8 // 2, w8 // 2) - 0.5) * 4,
        "params": r(1, 768, h8 // 2, w8 // 2) * 2 - 1,
    }


@torch.no_grad()
def make_modules(model):
    m = model.double().eval()
    inp = module_inputs()
    out = {}
    out["encoder"] = m.encoder(inp["x"], inp["ctx"], inp["q_enc"])
    out["hyper_encoder"] = m.hyper_encoder(out["encoder"])
    out["hyper_decoder"] = m.hyper_decoder(inp["z_hat"])
    out["temporal_prior_encoder"] = m.temporal_prior_encoder(inp["memory"], inp["q_feat"])
    out["prior_fusion"] = m.y_prior_fusion(out["hyper_decoder"], out["temporal_prior_encoder"])
    reduced = m.y_spatial_prior_reduction(inp["params"])
    out["reduction"] = reduced
    for k in (1, 2, 3):
        ad = getattr(m, f"y_spatial_prior_adaptor_{k}")
        out[f"spatial_prior_{k}"] = m.y_spatial_prior(ad(inp["y_hat"], reduced))
    out["decoder"] = m.decoder(inp["y_hat"], inp["ctx"], inp["q_dec"])
    recon = m.recon_head(inp["feature"])
    for i, r in enumerate(recon):
        out[f"recon_{i}"] = r
    out["recon_reset"] = m.recon_head(inp["feature"], for_reset=True)
    out["feature_adaptor_i"] = m.feature_adaptor_i(inp["feature_i"])
    out["feature_adaptor_m"] = m.feature_adaptor_m(inp["memory"], inp["feature"])
    out["feature_extractor"] = m.feature_extractor(inp["memory"])
    np.savez_compressed(os.path.join(HERE, "modules_golden.npz"),
                        **{k: v.float().numpy() for k, v in out.items()})
    m.half()  # leave the caller's model in a usable dtype
    m.float()
