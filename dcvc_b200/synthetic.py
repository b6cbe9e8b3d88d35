"""Seeded synthetic YUV420 content standing in for the reference's test sequences.

The reference measures on UVG / MCL-JCV / HEVC sequences (test_cfg/all_yuv420.json); none are
available, so the workloads use this generator:

* intra frame (seed 1): Y = 128 + 60 * mean of 4 random-phase 2D sinusoids (periods 16-128 px)
  + N(0, 3^2), clipped to [0, 255]; U/V the same construction at half resolution, amplitude 20.
* video chunk (seed 2): per frame t, the intra-style sinusoid field, plus a 256 x 256
  random-texture patch translating by (2, 1) px per frame, plus a global luma ramp drifting
  0.5 per frame, plus N(0, 2^2).

`to_model_input` converts frames as the reference harness does (test_video.py:69-123): UV
nearest-upsampled to 4:4:4, frames concatenated along channels, FP16, / 255, - 0.5.
"""
import numpy as np
import torch


def _sinusoids(rng, H, W, amplitude, base):
    yy, xx = np.mgrid[0:H, 0:W].astype(np.float64)
    field = np.zeros((H, W))
    for _ in range(4):
        period = rng.uniform(16, 128)
        theta = rng.uniform(0, np.pi)
        phase = rng.uniform(0, 2 * np.pi)
        f = 2 * np.pi / period
        field += np.sin(f * (np.cos(theta) * xx + np.sin(theta) * yy) + phase)
    return base + amplitude * field / 4.0


def intra_frame_yuv420(seed=1, H=256, W=256):
    rng = np.random.default_rng(seed)
    y = _sinusoids(rng, H, W, 60.0, 128.0) + rng.normal(0, 3.0, (H, W))
    u = _sinusoids(rng, H // 2, W // 2, 20.0, 128.0) + rng.normal(0, 3.0, (H // 2, W // 2))
    v = _sinusoids(rng, H // 2, W // 2, 20.0, 128.0) + rng.normal(0, 3.0, (H // 2, W // 2))
    q = lambda a: np.clip(np.round(a), 0, 255).astype(np.uint8)  # noqa: E731
    return q(y), q(u), q(v)


def video_chunk_yuv420(seed=2, H=1080, W=1920, frames=8, start=0):
    """List of `frames` (y, u, v) uint8 planes, frames start .. start + frames - 1."""
    rng = np.random.default_rng(seed)
    base_y = _sinusoids(rng, H, W, 60.0, 128.0)
    base_u = _sinusoids(rng, H // 2, W // 2, 20.0, 128.0)
    base_v = _sinusoids(rng, H // 2, W // 2, 20.0, 128.0)
    ps = min(256, H, W)
    patch = rng.uniform(0, 255, (ps, ps))
    patch_uv = rng.uniform(96, 160, (2, ps // 2, ps // 2))
    out = []
    for t in range(start, start + frames):
        nrng = np.random.default_rng(seed * 1000003 + t)
        y = base_y + 0.5 * t
        u = base_u.copy()
        v = base_v.copy()
        py = (H // 4 + 1 * t) % max(1, H - ps)
        px = (W // 4 + 2 * t) % max(1, W - ps)
        y[py:py + ps, px:px + ps] = patch
        u[py // 2:py // 2 + ps // 2, px // 2:px // 2 + ps // 2] = patch_uv[0]
        v[py // 2:py // 2 + ps // 2, px // 2:px // 2 + ps // 2] = patch_uv[1]
        y = y + nrng.normal(0, 2.0, (H, W))
        q = lambda a: np.clip(np.round(a), 0, 255).astype(np.uint8)  # noqa: E731
        out.append((q(y), q(u), q(v)))
    return out


def yuv420_to_444(y, u, v):
    """Nearest-neighbour chroma upsampling (transforms.py:69-80 with order 0)."""
    uu = np.repeat(np.repeat(u, 2, axis=0), 2, axis=1)[: y.shape[0], : y.shape[1]]
    vv = np.repeat(np.repeat(v, 2, axis=0), 2, axis=1)[: y.shape[0], : y.shape[1]]
    return np.stack([y, uu, vv], axis=0)


def to_model_input(frames, device="cuda"):
    """[1, 3 * len(frames), H, W] float16 channels-last tensor, as get_src_frame builds it."""
    x = torch.from_numpy(np.concatenate([yuv420_to_444(*f) for f in frames], axis=0)[None])
    x = x.to(device=device).half()
    x = x / 255.0
    x = x - 0.5
    return x.contiguous(memory_format=torch.channels_last)


def padded_reference_frame(frame, pad_to=16, device="cuda"):
    """[1, 3, Hp, Wp] model-domain frame, replicate-padded to a multiple of `pad_to`: the stand-in
    for the intra model's reconstruction that seeds the temporal context."""
    x = to_model_input([frame], device=device)
    H, W = x.shape[2], x.shape[3]
    ph, pw = (-H) % pad_to, (-W) % pad_to
    if ph or pw:
        x = torch.nn.functional.pad(x.float(), (0, pw, 0, ph), mode="replicate").half()
    return x.contiguous(memory_format=torch.channels_last)


def padding_for(H, W, p=16):
    """(padding_right, padding_bottom) as get_padding_size (common_model.py:103-108)."""
    return (W + p - 1) // p * p - W, (H + p - 1) // p * p - H
