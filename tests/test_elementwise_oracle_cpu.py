"""The NumPy FP16 oracle of the layout kernels agrees with PyTorch's pixel_(un)shuffle, which the
reference modules use (layers.py, video_model_ht.py); the quantiser oracle obeys the reference's
invariants (symbols in [-128, 127], skipped positions zero, restore inverts quantise)."""
import os
import sys

import numpy as np
import torch

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(__file__)), "oracle"))
import elementwise_oracle as O  # noqa: E402


def test_unshuffle_matches_torch():
    rng = np.random.default_rng(0)
    x = rng.standard_normal((64, 48, 3)).astype(np.float16)
    ref = torch.nn.functional.pixel_unshuffle(torch.from_numpy(x).permute(2, 0, 1)[None].float(), 8)
    ref = ref[0].permute(1, 2, 0).reshape(-1, 192).numpy().astype(np.float16)
    assert np.array_equal(O.pad_unshuffle8(x, 0, 0), ref)
    back = O.shuffle8_clamp(np.clip(ref, -0.5, 0.5).astype(np.float16), 8, 6)
    assert np.array_equal(back, np.clip(x, -0.5, 0.5).astype(np.float16))


def test_space_to_depth_matches_torch_order():
    rng = np.random.default_rng(1)
    H, W, C = 8, 6, 16
    x = rng.standard_normal((H * W, C)).astype(np.float16)
    t = torch.nn.functional.pixel_unshuffle(torch.from_numpy(x).view(H, W, C).permute(2, 0, 1)[None].float(), 2)
    t = t[0].permute(1, 2, 0).reshape(-1, 4 * C).numpy()  # channel c*4 + dy*2 + dx
    s2d = O.space_to_depth2(x, H, W).astype(np.float32)     # channel (dy*2 + dx)*C + c
    perm = np.array([(s % 4) * C + s // 4 for s in range(4 * C)])
    assert np.array_equal(s2d[:, perm], t)


def test_quantise_restore_round_trip():
    rng = np.random.default_rng(2)
    H, W, C = 6, 10, 256
    M = H * W
    y = (rng.standard_normal((M, C)) * 5).astype(np.float16)
    scales = np.abs(rng.standard_normal((M, C))).astype(np.float16)
    means = rng.standard_normal((M, C)).astype(np.float16)
    qd = rng.uniform(0.2, 2, (M, C)).astype(np.float16)
    yq = np.zeros((M, C), np.float16)
    yh = np.zeros((M, C), np.float16)
    rh = np.zeros((M, C), np.float16)
    for p in range(4):
        mode = 0 if p == 0 else (2 if p == 3 else 1)
        yq_p, yh = O.quantize_phase(p, mode, y, scales, means, qd, 0.15, yq, yh, H, W)
        q_only = O.quantize_phase(p, 0, y, scales, means, qd, 0.15, yq, yh, H, W)[0]
        rh = O.restore_phase(p, mode, q_only, means, qd, rh, H, W)
        yq = yq_p
    assert np.array_equal(yh.view(np.uint16), rh.view(np.uint16))
    assert yq.min() >= -128 and yq.max() <= 127
    assert (yq[scales <= np.float16(0.15)] == 0).all()
