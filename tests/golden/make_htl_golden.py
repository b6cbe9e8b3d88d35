"""Generates the HT-L golden fixtures under tests/golden/ from the reference itself.

Run here, where the reference sources exist (the reference checkout given by --ref or the DCVC_REFERENCE environment variable):

    python tests/golden/make_htl_golden.py [--ref <reference checkout>]

Outputs (small, committed):
  weights_htl_seed0.json   fingerprints of the reference DMC(ModelStructure.HTL) state dict for
                           torch.manual_seed(0)
  htl_modules_golden.npz   reference HT-L sub-network outputs for seeded inputs (float64)
"""
import argparse
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

# 64 x 64 frames: H8 x W8 = 8 x 8, y level 4 x 4, z level 1 x 1
H, W = 64, 64


def htl_module_inputs():
    import torch
    g = torch.Generator().manual_seed(2026)
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


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("DCVC_REFERENCE"),
                    help="reference checkout (default: $DCVC_REFERENCE)")
    args = ap.parse_args()
    if not args.ref:
        ap.error("give --ref or set DCVC_REFERENCE to the reference checkout")
    sys.path.insert(0, args.ref)
    import torch
    from src.models.video_model_ht import DMC
    from src.utils.common import ModelStructure
    from make_golden import fingerprint

    torch.manual_seed(0)
    model = DMC(ModelStructure.HTL)
    sd = {k: v.clone() for k, v in model.state_dict().items()}
    with open(os.path.join(HERE, "weights_htl_seed0.json"), "w") as f:
        json.dump(fingerprint(sd), f)
    m = model.double().eval()
    inp = htl_module_inputs()
    out = {}
    with torch.no_grad():
        out["encoder"] = m.encoder(inp["x"], inp["ctx"], inp["q_enc"])
        out["hyper_encoder"] = m.hyper_encoder(out["encoder"])
        out["hyper_decoder"] = m.hyper_decoder(inp["z_hat"])
        out["temporal_prior_encoder"] = m.temporal_prior_encoder(inp["memory"], inp["q_feat"])
        out["prior_fusion"] = m.y_prior_fusion(out["hyper_decoder"], out["temporal_prior_encoder"])
        reduced = m.y_spatial_prior_reduction(inp["params"])
        out["reduction"] = reduced
        for k in (1, 2, 3):
            ad = getattr(m, f"y_spatial_prior_adaptor_{k}")
            out[f"spatial_prior_{k}"] = m.y_spatial_prior(ad(torch.cat((inp["y_hat"], reduced), 1)))
        out["decoder"] = m.decoder(inp["y_hat"], inp["ctx"], inp["q_dec"])
        for i, r in enumerate(m.recon_head(inp["feature"])):
            out[f"recon_{i}"] = r
        out["recon_reset"] = m.recon_head(inp["feature"], for_reset=True)
        out["feature_adaptor_i"] = m.feature_adaptor_i(inp["feature_i"])
        out["feature_adaptor_m"] = m.feature_adaptor_m(inp["memory"], inp["feature"])
        out["feature_extractor"] = m.feature_extractor(inp["memory"])
    np.savez_compressed(os.path.join(HERE, "htl_modules_golden.npz"),
                        **{k: v.float().numpy() for k, v in out.items()})
    print("HT-L golden fixtures written to", HERE)


if __name__ == "__main__":
    sys.path.insert(0, HERE)
    main()
