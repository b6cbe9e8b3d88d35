"""Generates tests/golden/yuv_golden.npz from the reference's own YUV conversions.

Run here, where the reference sources exist (the reference checkout given by --ref or the DCVC_REFERENCE environment variable):

    python tests/golden/make_yuv_golden.py [--ref <reference checkout>]

The model input is built as get_src_frame does (test_video.py:69-123): ycbcr420_to_444_np on
the uint8 planes, torch.from_numpy, .half(), / 255.0, - 0.5.  The reconstruction planes are built
as the decoded-frame writer does (test_video.py:355-362): yuv_444_to_420(x_hat + 0.5), Y
clamp(* 255).round().byte(), UV clamp(* 255).byte().  Both on CPU torch.
"""
import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
H, W, F = 18, 26, 2       # picture size and frames
HP, WP = 32, 32           # padded reconstruction size


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("DCVC_REFERENCE"),
                    help="reference checkout (default: $DCVC_REFERENCE)")
    args = ap.parse_args()
    if not args.ref:
        ap.error("give --ref or set DCVC_REFERENCE to the reference checkout")
    sys.path.insert(0, args.ref)
    import torch
    from src.utils.transforms import ycbcr420_to_444_np, yuv_444_to_420

    rng = np.random.default_rng(2026)
    planes = rng.integers(0, 256, F * H * W * 3 // 2).astype(np.uint8)
    fb = H * W * 3 // 2
    xs = []
    for f in range(F):
        fr = planes[f * fb:(f + 1) * fb]
        y = fr[:H * W].reshape(1, H, W)
        uv = fr[H * W:].reshape(2, H // 2, W // 2)
        xs.append(torch.from_numpy(ycbcr420_to_444_np(y, uv)).unsqueeze(0))
    x = torch.cat(xs, dim=1).half()
    x = x / 255.0
    x = x - 0.5
    model_input = x[0].permute(1, 2, 0).numpy()  # [H, W, 3F]

    # reconstructions: values in [-0.5, 0.5] with exact half-steps near the rounding points
    g = torch.Generator().manual_seed(7)
    x_hat = ((torch.rand(F, 3, HP, WP, generator=g) - 0.5)).half()
    x_hat[:, :, 0, :8] = torch.tensor([-0.5, 0.5, 0.0, 1 / 510, -1 / 510, 0.25, 0.3, -0.49]).half()
    recs = []
    for f in range(F):
        xh = x_hat[f:f + 1, :, :H, :W]
        y_rec, uv_rec = yuv_444_to_420(xh + 0.5)
        y_rec = torch.clamp(y_rec * 255, 0, 255).round().byte().squeeze(0).numpy()
        uv_rec = torch.clamp(uv_rec * 255, 0, 255).byte().squeeze(0).numpy()
        recs += [y_rec.reshape(-1), uv_rec.reshape(-1)]
    np.savez_compressed(os.path.join(HERE, "yuv_golden.npz"), planes=planes,
                        model_input=model_input, x_hat=x_hat.permute(0, 2, 3, 1).numpy(),
                        rec_planes=np.concatenate(recs), shape=np.array([H, W, F, HP, WP]))
    print("YUV golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
