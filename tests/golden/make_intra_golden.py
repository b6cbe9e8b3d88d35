"""Generates the intra-model golden fixtures under tests/golden/ from the reference itself.

Run here, where the reference sources exist (the reference checkout given by --ref or the DCVC_REFERENCE environment variable) and oracle/_ref has been
built by `make -C oracle`:

    python tests/golden/make_intra_golden.py [--ref <reference checkout>]

Outputs (small, committed):
  weights_intra_seed0.json    fingerprints of the reference DMCI() state dict for torch.manual_seed(0)
  intra_modules_golden.npz    reference DMCI sub-network outputs for seeded inputs (float64)
  rans_segments_golden.npz    the reference coder's bytes for payloads of four y segments + z (the
                              intra worker's call sequence) at several ec_parallel values
"""
import argparse
import ctypes
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))

# 128 x 64 frames: H8 x W8 = 16 x 8, y level 8 x 4, z level 2 x 1
H, W = 128, 64
SEG_QP = 37
SEG_COUNTS = (5003, 0, 1, 40000)
SEG_ECPS = (1, 2, 3, 4, 7, 8)


def intra_module_inputs():
    import torch
    g = torch.Generator().manual_seed(2025)
    r = lambda *s: torch.rand(*s, generator=g, dtype=torch.float64)  # noqa: E731
    h16, w16 = H // 16, W // 16
    return {
        "x": r(1, 3, H, W) - 0.5,
        "q_enc": r(1, 384, 1, 1) + 0.5,
        "q_dec": r(1, 384, 1, 1) + 0.5,
        "z_hat": torch.round((r(1, 128, h16 // 4, w16 // 4) - 0.5) * 8),
        "y_hat": (r(1, 256, h16, w16) - 0.5) * 4,
        "params": r(1, 512, h16, w16) * 2 - 1,
    }


def segment_inputs():
    """Four y segments (coding order) and the z symbols, seeded."""
    rng = np.random.default_rng(77)
    segs = []
    for n in SEG_COUNTS:
        v = np.clip(np.round(rng.laplace(0, 3, n)), -128, 127).astype(np.int64)
        idx = rng.integers(0, 128, n)
        segs.append(((v << 8) + idx).astype(np.int16))
    z = np.clip(np.round(rng.laplace(0, 2, 128 * 6)), -64, 63).astype(np.int8)
    return segs, z


def make_segments(qy, ly, qz, lz):
    lib = ctypes.PyDLL(os.path.join(ROOT, "oracle", "_ref", "librans_ref.so"))
    p = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    segs, z = segment_inputs()
    counts = np.array([s.size for s in segs], np.int32)
    y_all = np.ascontiguousarray(np.concatenate(segs), np.int16)
    out = {"counts": counts, "qp": np.int32(SEG_QP)}
    for ecp in SEG_ECPS:
        cap = (y_all.size + z.size) * 4 + 4096
        buf = np.zeros(cap, np.uint8)
        n = lib.ref_encode_segments(p(qz), p(lz), qz.shape[0], qz.shape[1], p(qy), p(ly),
                                    qy.shape[0], qy.shape[1], p(y_all), p(counts), counts.size,
                                    p(z), z.size, SEG_QP * 128, 128, ecp, p(buf), cap)
        assert n > 0
        out[f"bytes_{ecp}"] = buf[:n].copy()
    np.savez_compressed(os.path.join(HERE, "rans_segments_golden.npz"), **out)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("DCVC_REFERENCE"),
                    help="reference checkout (default: $DCVC_REFERENCE)")
    args = ap.parse_args()
    if not args.ref:
        ap.error("give --ref or set DCVC_REFERENCE to the reference checkout")
    sys.path.insert(0, args.ref)
    import torch
    from src.models.image_model import DMCI
    from make_golden import fingerprint

    torch.manual_seed(0)
    model = DMCI()
    sd = {k: v.clone() for k, v in model.state_dict().items()}
    with open(os.path.join(HERE, "weights_intra_seed0.json"), "w") as f:
        json.dump(fingerprint(sd), f)
    m = model.double().eval()
    inp = intra_module_inputs()
    out = {}
    with torch.no_grad():
        out["encoder"] = m.enc(inp["x"], inp["q_enc"])
        out["hyper_encoder"] = m.hyper_enc(out["encoder"])
        out["hyper_decoder"] = m.hyper_dec(inp["z_hat"])
        out["prior_fusion"] = m.y_prior_fusion(out["hyper_decoder"])
        reduced = m.y_spatial_prior_reduction(inp["params"])
        out["reduction"] = reduced
        for k in (1, 2, 3):
            ad = getattr(m, f"y_spatial_prior_adaptor_{k}")
            out[f"spatial_prior_{k}"] = m.y_spatial_prior(ad(torch.cat((inp["y_hat"], reduced), 1)))
        out["decoder"] = m.dec(inp["y_hat"], inp["q_dec"])
    np.savez_compressed(os.path.join(HERE, "intra_modules_golden.npz"),
                        **{k: v.float().numpy() for k, v in out.items()})
    g = np.load(os.path.join(HERE, "cdf_tables.npz"))
    make_segments(*[np.ascontiguousarray(g[k], np.int32) for k in ("qy", "ly", "qz", "lz")])
    print("intra golden fixtures written to", HERE)


if __name__ == "__main__":
    sys.path.insert(0, HERE)
    main()
