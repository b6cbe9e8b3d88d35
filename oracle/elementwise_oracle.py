"""ORACLE (test infrastructure only; never imported by the product).

NumPy restatements of the reference's FP16 elementwise, layout and quantisation kernels, with
the reference's arithmetic: every FP16 op is evaluated in float32 and rounded once to float16
(at::Half semantics), max/min are the NaN-ignoring FP16 max/min (np.fmax/np.fmin), rounding is
half away from zero (roundf), comparisons are false for NaN.  Arrays are NHWC: [H, W, C] or
[M, C] float16.  Each function cites the reference kernel it restates
(src/layers/extensions/inference/elementwise/*.cu).
"""
import numpy as np

F16, F32 = np.float16, np.float32
MASK_PERM = (0, 3, 2, 1)


def _h(x):
    return np.asarray(x, dtype=F32).astype(F16)


def hadd(a, b):
    return _h(a.astype(F32) + b.astype(F32))


def hsub(a, b):
    return _h(a.astype(F32) - b.astype(F32))


def hmul(a, b):
    return _h(a.astype(F32) * b.astype(F32))


def roundf(a):
    """roundf: half away from zero, keeping the sign of zero."""
    f = a.astype(F32)
    return np.copysign(np.floor(np.abs(f) + F32(0.5)), f)


def pad_unshuffle8(x, pad_b, pad_r):
    """cat_and_pad.cu:7-51 -> [H8 * W8, 64 C]."""
    H, W, C = x.shape
    H8, W8 = (H + pad_b) // 8, (W + pad_r) // 8
    hh = np.minimum(np.arange(H8 * 8), H - 1)
    ww = np.minimum(np.arange(W8 * 8), W - 1)
    p = x[hh][:, ww]  # [8 H8, 8 W8, C]
    p = p.reshape(H8, 8, W8, 8, C).transpose(0, 2, 4, 1, 3)  # h8, w8, c, dy, dx
    return p.reshape(H8 * W8, C * 64)


def shuffle8_clamp(x, H8, W8):
    """shuffle.cu:40-131 (clamp to [-0.5, 0.5]) -> [8 H8, 8 W8, C]."""
    C = x.shape[1] // 64
    p = x.reshape(H8, W8, C, 8, 8).transpose(0, 3, 1, 4, 2).reshape(8 * H8, 8 * W8, C)
    p = np.fmax(p, F16(-0.5))
    return np.fmin(p, F16(0.5))


def space_to_depth2(x, H, W):
    C = x.shape[1]
    p = x.reshape(H // 2, 2, W // 2, 2, C).transpose(0, 2, 1, 3, 4)
    return p.reshape((H // 2) * (W // 2), 4 * C)


def im2col3x3s2(x, H, W):
    C = x.shape[1]
    g = np.zeros((H + 2, W + 2, C), F16)
    g[1:-1, 1:-1] = x.reshape(H, W, C)
    cols = []
    for ky in range(3):
        for kx in range(3):
            cols.append(g[ky:ky + H:2, kx:kx + W:2])
    return np.concatenate(cols, axis=2).reshape((H // 2) * (W // 2), 9 * C)


def replicate_pad(x, H, W, pad_b, pad_r):
    C = x.shape[1]
    g = x.reshape(H, W, C)
    hh = np.minimum(np.arange(H + pad_b), H - 1)
    ww = np.minimum(np.arange(W + pad_r), W - 1)
    return g[hh][:, ww].reshape(-1, C)


def round_z(z):
    """stream.cu:862-894 -> (z_hat FP16, int8)."""
    v = _h(roundf(z))
    v = np.fmax(v, F16(-64))
    v = np.fmin(v, F16(63))
    return v, v.astype(F32).astype(np.int8)


def mul_channel(x, q):
    return hmul(x, q[None, :])


def div_clamp(y, q):
    """stream.cu:422-452: y * rcp(max(q, 0.5)), the reciprocal rounded from float32 1/q."""
    qc = np.fmax(q, F16(0.5))
    r = _h(F32(1.0) / qc.astype(F32))
    return hmul(y, r)


def mask(phase, H, W, C):
    q = np.arange(C) // (C // 4)
    pos = q ^ MASK_PERM[phase]
    hw = (np.arange(H)[:, None] % 2) * 2 + (np.arange(W)[None, :] % 2)
    return (hw[:, :, None] == pos[None, None, :]).reshape(H * W, C)


def quantize_phase(phase, mode, y, scales, means, q_dec, thr, y_q_prev, y_hat_prev, H, W):
    """stream.cu:548-683 -> (y_q, y_hat)."""
    C = y.shape[1]
    on = mask(phase, H, W, C)
    z = F16(0)
    thr = F16(thr)
    s_hat = np.where(on, scales, z)
    m_hat = np.where(on, means, z)
    res = np.where(on, hsub(y, m_hat), z)
    q = _h(roundf(res))
    with np.errstate(invalid="ignore"):
        q = np.where(s_hat > thr, q, z)
    q = np.fmax(np.fmin(q, F16(127)), F16(-128))
    yh = hadd(q, m_hat)
    if mode == 0:
        return q, yh
    yq = hadd(y_q_prev, q)
    yh = hadd(yh, y_hat_prev)
    if mode == 2:
        yh = hmul(yh, np.fmax(q_dec, F16(0.5)))
    return yq, yh


def restore_phase(phase, mode, y_q, means, q_dec, y_hat_prev, H, W):
    """stream.cu:685-760 -> y_hat."""
    C = y_q.shape[1]
    on = mask(phase, H, W, C)
    t = np.where(on, hadd(y_q, means), F16(0))
    if mode >= 1:
        t = hadd(t, y_hat_prev)
    if mode == 2:
        t = hmul(t, np.fmax(q_dec, F16(0.5)))
    return t


def build_index(encode, y_q, scales, thr, lut):
    """stream.cu:89-173 in NHWC order -> (sym int16 or idx uint8, cond uint8)."""
    s = scales.reshape(-1)
    idx = lut[s.view(np.uint16)]
    with np.errstate(invalid="ignore"):
        cond = (s > F16(thr)).astype(np.uint8)
    if not encode:
        return idx, cond
    q = np.floor(y_q.reshape(-1).astype(F32)).astype(np.int32)
    return (q * 256 + idx.astype(np.int32)).astype(np.int16), cond


def compact(src, cond):
    """conditional_index_part1/2 (stream.cu:175-357)."""
    keep = cond.astype(bool)
    return src[keep], int(keep.sum())


def recover(dec, cond):
    """stream.cu:359-420."""
    keep = cond.astype(bool)
    out = np.zeros(cond.size, F16)
    out[keep] = dec[: int(keep.sum())].astype(F32).astype(F16)
    return out
