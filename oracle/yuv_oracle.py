"""ORACLE (test infrastructure only; never imported by the product).

NumPy restatement of the reference test harness's YUV 4:2:0 conversions, pinned by
tests/golden/yuv_golden.npz (made from the reference's own functions by
tests/golden/make_yuv_golden.py):

* model input (test_video.py:69-123, get_src_frame): ycbcr420_to_444_np (transforms.py:69-80,
  scipy zoom with order 0 = each chroma sample repeated 2 x 2), then in FP16: x / 255.0 - 0.5,
  every operation computed in FP32 and rounded to FP16;
* decoded-frame writer (test_video.py:355-362, yuv_444_to_420 transforms.py:83-90): x = x_hat +
  0.5 in FP16; Y = round(clamp(FP16(x * 255), 0, 255)); chroma = avg_pool2d 2 x 2 (FP32 sum in
  row-major order, / 4, rounded to FP16), then trunc(clamp(FP16(c * 255), 0, 255)).
"""
import numpy as np


def _h(x):
    return np.asarray(x, dtype=np.float32).astype(np.float16)


def yuv420_to_input(planes, frames, H, W):
    """planes: uint8 [frames * H * W * 3 / 2] (I420 frames back to back) -> float16 [H, W, 3F]."""
    fb = H * W * 3 // 2
    out = np.empty((H, W, 3 * frames), dtype=np.float16)
    for f in range(frames):
        fr = planes[f * fb:(f + 1) * fb]
        y = fr[:H * W].reshape(H, W)
        u = fr[H * W:H * W + H * W // 4].reshape(H // 2, W // 2)
        v = fr[H * W + H * W // 4:].reshape(H // 2, W // 2)
        for c, p in enumerate((y, np.repeat(np.repeat(u, 2, 0), 2, 1),
                               np.repeat(np.repeat(v, 2, 0), 2, 1))):
            a = _h(p.astype(np.float32) / np.float32(255.0))
            out[:, :, 3 * f + c] = _h(a.astype(np.float32) - np.float32(0.5))
    return out


def frames_to_yuv420(frames, H, W):
    """frames: list of float16 [Hp, Wp, 3] pictures -> uint8 I420 planes (cropped to H x W)."""
    out = []
    for fr in frames:
        x = _h(fr[:H, :W].astype(np.float32) + np.float32(0.5)).astype(np.float32)
        y = np.clip(_h(x[:, :, 0] * np.float32(255.0)).astype(np.float32), 0, 255)
        out.append(np.rint(y).astype(np.uint8).reshape(-1))
        for c in (1, 2):
            a = x[:, :, c]
            s = ((a[0::2, 0::2] + a[0::2, 1::2]) + a[1::2, 0::2]) + a[1::2, 1::2]
            m = _h(s / np.float32(4.0)).astype(np.float32)
            t = np.clip(_h(m * np.float32(255.0)).astype(np.float32), 0, 255)
            out.append(np.trunc(t).astype(np.uint8).reshape(-1))
    return np.concatenate(out)
