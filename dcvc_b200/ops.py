"""Thin torch-facing wrappers over the kernel-level C ABI (device tensors in, device tensors out).

These exist for tests and for callers that compose their own graphs; the codec runtime itself
drives the kernels from C++.  Every wrapper runs the sm_100a kernel through libdcvc_b200.so on
the current CUDA stream; nothing here falls back to PyTorch math.
"""
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
