"""Thin torch-facing wrappers over the kernel-level C ABI (device tensors in, device tensors out).

These exist for tests and for callers that compose their own graphs; the codec runtime itself
drives the kernels from C++.  Every wrapper runs the sm_100a kernel through libdcvc_b200.so on
the current CUDA stream; nothing here falls back to PyTorch math.
"""
import ctypes

import torch

from . import _native as N

_DT = {torch.float16: N.F16, torch.bfloat16: N.BF16}


def _ptr(t):
    return None if t is None else t.data_ptr()


def _stream():
    return torch.cuda.current_stream().cuda_stream


def conv1x1(a, w, bias=None, epilogue=N.EPI_BIAS, res=None, res2=None, qscale=None, out=None,
            sub_w=0, sub_cout=0, block_n=0):
    """out = epilogue(a . w^T) for a: [M, K] (row pitch a.stride(0)), w: [N, K].

    bias is fp32 [N]; res/res2 are [M, N] views; qscale is [N] in the activation dtype.
    QUAD returns [M, N/4]; SUBPEL returns [4*M, sub_cout] (the 2x pixel-shuffled grid).
    """
    assert a.dim() == 2 and a.stride(1) == 1 and w.is_contiguous()
    M, K = a.shape
    Nn = w.shape[0]
    if out is None:
        if epilogue == N.EPI_QUAD:
            out = torch.empty((M, Nn // 4), dtype=a.dtype, device=a.device)
        elif epilogue == N.EPI_SUBPEL:
            out = torch.empty((4 * M, sub_cout), dtype=a.dtype, device=a.device)
        else:
            out = torch.empty((M, Nn), dtype=a.dtype, device=a.device)
    N.check(N.lib.dcvc_conv1x1(
        _DT[a.dtype], epilogue, M, Nn, K, a.data_ptr(), a.stride(0), w.data_ptr(), _ptr(bias),
        _ptr(res), res.stride(0) if res is not None else 0,
        _ptr(res2), res2.stride(0) if res2 is not None else 0, _ptr(qscale),
        out.data_ptr(), out.stride(0), sub_w, sub_cout, block_n, _stream()), "dcvc_conv1x1")
    return out


def quantize_fp8(x, inv_scale, out=None):
    """E4M3 bytes of x * inv_scale (x: [M, C] float16 / bfloat16, row pitch x.stride(0)),
    saturating at +-448; returned as a torch.float8_e4m3fn tensor."""
    M, C = x.shape
    if out is None:
        out = torch.empty((M, C), dtype=torch.float8_e4m3fn, device=x.device)
    N.check(N.lib.dcvc_quantize_fp8(x.data_ptr(), _DT[x.dtype], x.stride(0), ctypes.c_float(inv_scale),
                                    out.data_ptr(), out.stride(0), M, C, _stream()),
            "dcvc_quantize_fp8")
    return out


def conv1x1_f8(a, w, wscale, bias, epilogue=N.EPI_BIAS, out=None, block_n=0):
    """The FP8 GEMM form: a [M, K] and w [N, K] float8_e4m3fn, wscale [N] fp32 (activation scale
    times weight-row scale), bias [N] fp32; returns bfloat16 epilogue(acc * wscale + bias)
    ([M, N/4] for the QUAD epilogue)."""
    assert a.dim() == 2 and a.stride(1) == 1 and w.is_contiguous()
    M, K = a.shape
    Nn = w.shape[0]
    if out is None:
        out = torch.empty((M, Nn // 4 if epilogue == N.EPI_QUAD else Nn), dtype=torch.bfloat16,
                          device=a.device)
    N.check(N.lib.dcvc_conv1x1_f8(epilogue, M, Nn, K, a.data_ptr(), a.stride(0), w.data_ptr(),
                                  wscale.data_ptr(), bias.data_ptr(), out.data_ptr(), out.stride(0),
                                  block_n, _stream()), "dcvc_conv1x1_f8")
    return out


def gemm_autotune(dtype, epilogue, M, Nn, K, sub_w=0, sub_cout=0):
    """Times every valid N tile width of one conv1x1 shape on the current stream and records the
    fastest for conv1x1(block_n=0) and the codecs.  Returns (block_n, microseconds per launch)."""
    bn, us = ctypes.c_int(), ctypes.c_float()
    N.check(N.lib.dcvc_gemm_autotune(_DT[dtype], epilogue, M, Nn, K, sub_w, sub_cout, _stream(),
                                     ctypes.byref(bn), ctypes.byref(us)), "dcvc_gemm_autotune")
    return bn.value, us.value


def gemm_autotune_enable(on=True):
    """Codecs tune each new GEMM shape on the first, eager run of a phase (before capture)."""
    N.check(N.lib.dcvc_gemm_autotune_enable(1 if on else 0), "dcvc_gemm_autotune_enable")


def gemm_tuned(dtype, epilogue, M, Nn, K, sub_w=0):
    """The recorded tile width of a shape, 0 if it has not been tuned."""
    bn = ctypes.c_int()
    N.check(N.lib.dcvc_gemm_tuned(_DT[dtype], epilogue, M, Nn, K, sub_w, ctypes.byref(bn)),
            "dcvc_gemm_tuned")
    return bn.value


def gemm_tuning_clear():
    N.check(N.lib.dcvc_gemm_tuning_clear(), "dcvc_gemm_tuning_clear")


def conv_ffn(x, w1, b1, w2, b2, qscale=None, out=None, block_n=0):
    """Fused ConvFFN: (quad(x . w1^T + b1) . w2^T + b2 + x) [* qscale] for x [M, C] fp16;
    w1 [4 cffn, C], w2 [C, cffn] fp16, b1 / b2 fp32."""
    assert x.dim() == 2 and x.stride(1) == 1 and w1.is_contiguous() and w2.is_contiguous()
    M, C = x.shape
    cffn = w2.shape[1]
    if out is None:
        out = torch.empty((M, C), dtype=x.dtype, device=x.device)
    N.check(N.lib.dcvc_conv_ffn(M, C, cffn, x.data_ptr(), x.stride(0), w1.data_ptr(),
                                b1.data_ptr(), w2.data_ptr(), b2.data_ptr(), _ptr(qscale),
                                out.data_ptr(), out.stride(0), block_n, _stream()),
            "dcvc_conv_ffn")
    return out


def dwconv3x3(x, H, W, w, out=None):
    """Depthwise 3x3 (pad 1, no bias) over an [H*W, C] NHWC tensor; w is fp32 [9, C]."""
    C = x.shape[1]
    if out is None:
        out = torch.empty_like(x)
    N.check(N.lib.dcvc_dwconv3x3(x.data_ptr(), H, W, C, x.stride(0), w.data_ptr(), out.data_ptr(),
                                 out.stride(0), _stream()), "dcvc_dwconv3x3")
    return out


def dwconv3x3_ex(x, H, W, w, img_h=0, out=None):
    """dwconv3x3 for FP16 or BF16 x over images of img_h rows stacked along H (0: one image)."""
    C = x.shape[1]
    if out is None:
        out = torch.empty_like(x)
    N.check(N.lib.dcvc_dwconv3x3_ex(_DT[x.dtype], x.data_ptr(), H, W, img_h, C, x.stride(0), w.data_ptr(),
                                    out.data_ptr(), out.stride(0), _stream()), "dcvc_dwconv3x3_ex")
    return out


def dw3x3_conv1x1_res(x, H, W, dw_w, w, bias, res, img_h=0, out=None):
    """(dwconv3x3_ex(x) . w^T + bias + res) in one launch: x [H*W, K], dw_w fp32 [9, K],
    w [N, K], bias fp32 [N], res [H*W, N] (row pitches from the tensors)."""
    M, K = x.shape
    Nn = w.shape[0]
    assert M == H * W and w.shape[1] == K and w.is_contiguous() and dw_w.is_contiguous()
    if out is None:
        out = torch.empty((M, Nn), dtype=x.dtype, device=x.device)
    N.check(N.lib.dcvc_dw3x3_conv1x1_res(_DT[x.dtype], H, W, img_h, x.data_ptr(), x.stride(0), dw_w.data_ptr(),
                                         K, w.data_ptr(), Nn, bias.data_ptr(), res.data_ptr(), res.stride(0),
                                         out.data_ptr(), out.stride(0), _stream()), "dcvc_dw3x3_conv1x1_res")
    return out


# ----------------------------------------------------------------------------- elementwise

def _sig(name, args):
    f = getattr(N.lib, name)
    f.restype = ctypes.c_int
    f.argtypes = args
    return f


_i, _v, _f = ctypes.c_int, ctypes.c_void_p, ctypes.c_float
_sig("dcvc_pad_unshuffle8", [_v, _i, _i, _i, _i, _i, _i, _v, _i, _v])
_sig("dcvc_shuffle8_clamp", [_v, _i, _i, _i, _i, _v, _v])
_sig("dcvc_space_to_depth2", [_v, _i, _i, _i, _i, _v, _v])
_sig("dcvc_im2col3x3s2", [_v, _i, _i, _i, _i, _v, _v])
_sig("dcvc_replicate_pad", [_v, _i, _i, _i, _i, _i, _i, _v, _v])
_sig("dcvc_crop", [_v, _i, _i, _i, _i, _i, _v, _i, _v])
_sig("dcvc_round_z", [_v, _i, _v, _v, _v])
_sig("dcvc_int8_to_half", [_v, _i, _v, _v])
_sig("dcvc_mul_channel", [_v, _i, _i, _i, _v, _v, _i, _v])
_sig("dcvc_div_clamp", [_v, _i, _i, _i, _v, _i, _v])
_sig("dcvc_quantize_phase", [_i, _i, _v, _i, _v, _i, _v, _i, _v, _i, _f, _v, _i, _v, _i, _i, _i, _i, _v])
_sig("dcvc_restore_phase", [_i, _i, _v, _i, _v, _i, _v, _i, _v, _i, _i, _i, _i, _v])
_sig("dcvc_build_index", [_i, _v, _i, _v, _i, _f, _v, _i, _i, _v, _v, _v, _v])
_sig("dcvc_compact_blocks", [_i])
_sig("dcvc_compact", [_v, _i, _v, _i, _v, _v, _v, _v])
_sig("dcvc_recover", [_v, _v, _v, _i, _v, _v])
_sig("dcvc_scale_index_table", [_v])
_sig("dcvc_scale_index_table_device", [_v, _v])
_sig("dcvc_quantize_fp8", [_v, _i, _i, ctypes.c_float, _v, _i, _i, _i, _v])
_sig("dcvc_conv1x1_f8", [_i, _i, _i, _i, _v, _i, _v, _v, _v, _v, _i, _i, _v])
_sig("dcvc_yuv420_to_input", [_v, _i, _i, _i, _v, _i, _v])
_sig("dcvc_frames_to_yuv420", [ctypes.POINTER(_v), _i, _i, _i, _i, _i, _v, _v])


def pad_unshuffle8(x, pad_b, pad_r, out=None):
    """x: [H, W, C] fp16 (dense) -> [(H+pad_b)/8 * (W+pad_r)/8, 64 C]."""
    H, W, C = x.shape
    if out is None:
        out = torch.empty(((H + pad_b) // 8) * ((W + pad_r) // 8), 64 * C, dtype=x.dtype, device=x.device)
    N.check(N.lib.dcvc_pad_unshuffle8(x.data_ptr(), H, W, C, C, pad_b, pad_r, out.data_ptr(),
                                      out.stride(0), _stream()), "pad_unshuffle8")
    return out


def shuffle8_clamp(x, H8, W8):
    """x: [H8*W8, 64 C] -> [8 H8, 8 W8, C]."""
    C = x.shape[1] // 64
    out = torch.empty(8 * H8, 8 * W8, C, dtype=x.dtype, device=x.device)
    N.check(N.lib.dcvc_shuffle8_clamp(x.data_ptr(), H8, W8, C, x.stride(0), out.data_ptr(),
                                      _stream()), "shuffle8_clamp")
    return out


def space_to_depth2(x, H, W):
    C = x.shape[1]
    out = torch.empty((H // 2) * (W // 2), 4 * C, dtype=x.dtype, device=x.device)
    N.check(N.lib.dcvc_space_to_depth2(x.data_ptr(), H, W, C, x.stride(0), out.data_ptr(), _stream()),
            "space_to_depth2")
    return out


def im2col3x3s2(x, H, W):
    C = x.shape[1]
    out = torch.empty((H // 2) * (W // 2), 9 * C, dtype=x.dtype, device=x.device)
    N.check(N.lib.dcvc_im2col3x3s2(x.data_ptr(), H, W, C, x.stride(0), out.data_ptr(), _stream()),
            "im2col3x3s2")
    return out


def replicate_pad(x, H, W, pad_b, pad_r):
    C = x.shape[1]
    out = torch.empty((H + pad_b) * (W + pad_r), C, dtype=x.dtype, device=x.device)
    N.check(N.lib.dcvc_replicate_pad(x.data_ptr(), H, W, C, x.stride(0), pad_b, pad_r,
                                     out.data_ptr(), _stream()), "replicate_pad")
    return out


def crop(x, Wx, H, W):
    C = x.shape[1]
    out = torch.empty(H * W, C, dtype=x.dtype, device=x.device)
    N.check(N.lib.dcvc_crop(x.data_ptr(), Wx, x.stride(0), H, W, C, out.data_ptr(), out.stride(0),
                            _stream()), "crop")
    return out


def round_z(z):
    z_hat = torch.empty_like(z)
    z_i8 = torch.empty(z.shape, dtype=torch.int8, device=z.device)
    N.check(N.lib.dcvc_round_z(z.data_ptr(), z.numel(), z_hat.data_ptr(), z_i8.data_ptr(), _stream()),
            "round_z")
    return z_hat, z_i8


def int8_to_half(x):
    out = torch.empty(x.shape, dtype=torch.float16, device=x.device)
    N.check(N.lib.dcvc_int8_to_half(x.data_ptr(), x.numel(), out.data_ptr(), _stream()), "int8_to_half")
    return out


def mul_channel(x, q):
    M, C = x.shape
    out = torch.empty_like(x)
    N.check(N.lib.dcvc_mul_channel(x.data_ptr(), M, C, x.stride(0), q.data_ptr(), out.data_ptr(),
                                   out.stride(0), _stream()), "mul_channel")
    return out


def div_clamp_(y, q):
    M, C = y.shape
    N.check(N.lib.dcvc_div_clamp(y.data_ptr(), M, C, y.stride(0), q.data_ptr(), q.stride(0), _stream()),
            "div_clamp")
    return y


def quantize_phase(phase, mode, y, scales, means, q_dec, thr, y_q, y_hat, H, W):
    C = y.shape[1]
    N.check(N.lib.dcvc_quantize_phase(
        phase, mode, y.data_ptr(), y.stride(0), scales.data_ptr(), scales.stride(0), means.data_ptr(),
        means.stride(0), _ptr(q_dec), q_dec.stride(0) if q_dec is not None else 0, float(thr),
        y_q.data_ptr(), y_q.stride(0), y_hat.data_ptr(), y_hat.stride(0), H, W, C, _stream()),
        "quantize_phase")


def restore_phase(phase, mode, y_q, means, q_dec, y_hat, H, W):
    C = y_q.shape[1]
    N.check(N.lib.dcvc_restore_phase(
        phase, mode, y_q.data_ptr(), y_q.stride(0), means.data_ptr(), means.stride(0), _ptr(q_dec),
        q_dec.stride(0) if q_dec is not None else 0, y_hat.data_ptr(), y_hat.stride(0), H, W, C,
        _stream()), "restore_phase")


def scale_index_table(device="cuda"):
    """The host-computed table (CPU restatement, double-precision logarithm)."""
    lut = torch.empty(65536, dtype=torch.uint8)
    N.check(N.lib.dcvc_scale_index_table(lut.data_ptr()), "scale_index_table")
    return lut.to(device)


def scale_index_table_device():
    """The table the codecs use: the reference's FP16 scale_to_index evaluated on the device."""
    lut = torch.empty(65536, dtype=torch.uint8, device="cuda")
    N.check(N.lib.dcvc_scale_index_table_device(lut.data_ptr(), _stream()),
            "scale_index_table_device")
    return lut


def build_index(encode, y_q, scales, thr, lut):
    M, C = scales.shape
    n = M * C
    sym = torch.empty(n, dtype=torch.int16, device=scales.device) if encode else None
    idx = None if encode else torch.empty(n, dtype=torch.uint8, device=scales.device)
    cond = torch.empty(n, dtype=torch.uint8, device=scales.device)
    N.check(N.lib.dcvc_build_index(
        1 if encode else 0, _ptr(y_q), y_q.stride(0) if y_q is not None else 0, scales.data_ptr(),
        scales.stride(0), float(thr), lut.data_ptr(), M, C, _ptr(sym), _ptr(idx), cond.data_ptr(),
        _stream()), "build_index")
    return (sym if encode else idx), cond


def compact(src, cond):
    n = src.numel()
    nb = N.lib.dcvc_compact_blocks(n)
    counts = torch.empty(nb, dtype=torch.int32, device=src.device)
    dst = torch.empty_like(src)
    total = torch.empty(1, dtype=torch.int32, device=src.device)
    N.check(N.lib.dcvc_compact(src.data_ptr(), src.element_size(), cond.data_ptr(), n,
                               counts.data_ptr(), dst.data_ptr(), total.data_ptr(), _stream()),
            "compact")
    return dst, total, counts


def recover(dec, cond, counts):
    n = cond.numel()
    out = torch.empty(n, dtype=torch.float16, device=cond.device)
    N.check(N.lib.dcvc_recover(dec.data_ptr(), cond.data_ptr(), counts.data_ptr(), n, out.data_ptr(),
                               _stream()), "recover")
    return out


# ----------------------------------------------------------------------------- YUV 4:2:0 I/O

def yuv420_to_input(planes, frames, H, W, out=None):
    """planes: uint8 CUDA tensor holding `frames` I420 frames back to back -> the model input
    [1, 3 * frames, H, W] float16 (channels last), as get_src_frame builds it."""
    if out is None:
        out = torch.empty((1, 3 * frames, H, W), dtype=torch.float16, device=planes.device,
                          memory_format=torch.channels_last)
    N.check(N.lib.dcvc_yuv420_to_input(planes.data_ptr(), frames, H, W, out.data_ptr(),
                                       out.stride(3), _stream()), "dcvc_yuv420_to_input")
    return out


def frames_to_yuv420(frames, H, W, out=None):
    """frames: list of [1, 3, Hp, Wp] float16 channels-last CUDA tensors (reconstructions in
    [-0.5, 0.5]) -> uint8 CUDA tensor of their I420 planes (cropped to H x W) back to back."""
    n = len(frames)
    if out is None:
        out = torch.empty(n * H * W * 3 // 2, dtype=torch.uint8, device=frames[0].device)
    for f in frames:
        if f.stride(1) != 1 or f.stride(3) != 3 or f.shape[1] != 3:
            raise ValueError("frames must be [1, 3, Hp, Wp] channels-last tensors")
    ptrs = (_v * n)(*[f.data_ptr() for f in frames])
    N.check(N.lib.dcvc_frames_to_yuv420(ptrs, n, H, W, frames[0].shape[3], 3, out.data_ptr(),
                                        _stream()), "dcvc_frames_to_yuv420")
    return out
