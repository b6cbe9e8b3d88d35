"""tcgen05 1x1-conv GEMM family vs a plain PyTorch fp32 reference of the same op.

Tolerance: FP16/BF16 operands with FP32 accumulation, output rounded once to the activation
type; we allow |err| <= atol + rtol*|ref| with (atol, rtol) = (2e-2, 1e-2) for f16 and
(6e-2, 2e-2) for bf16.
"""
import pytest
import torch

pytestmark = pytest.mark.gpu

TOL = {torch.float16: (2e-2, 1e-2), torch.bfloat16: (6e-2, 2e-2)}


def _wsilu(x):
    return x * torch.sigmoid(4.0 * x)


def _ref(epi, a, w, b, res=None, res2=None, q=None, sub_w=0, sub_cout=0):
    from dcvc_b200 import _native as N
    acc = a.float() @ w.float().t()
    if epi == N.EPI_SUBPEL:
        M = a.shape[0]
        H = M // sub_w
        t = acc.view(H, sub_w, 2, 2, sub_cout)  # (h, w, dy, dx, c)
        return t.permute(0, 2, 1, 3, 4).reshape(4 * M, sub_cout)
    acc = acc + b
    if epi == N.EPI_BIAS_WSILU:
        acc = _wsilu(acc)
    if epi in (N.EPI_BIAS_RES, N.EPI_BIAS_RES_Q, N.EPI_BIAS_RES2):
        acc = acc + res.float()
    if epi == N.EPI_BIAS_RES2:
        acc = acc + res2.float()
    if epi in (N.EPI_BIAS_RES_Q, N.EPI_BIAS_Q):
        acc = acc * q.float()
    if epi == N.EPI_QUAD:
        acc = _wsilu(acc).view(acc.shape[0], -1, 4).sum(-1)
    return acc


CASES = [
    # (epilogue name, M, N, K, dtype, block_n)
    ("EPI_BIAS", 1000, 256, 512, torch.float16, 0),
    ("EPI_BIAS", 32640, 512, 512, torch.float16, 0),
    ("EPI_BIAS", 8160, 768, 768, torch.float16, 0),
    ("EPI_BIAS", 510, 192, 256, torch.float16, 0),
    ("EPI_BIAS", 777, 128, 64, torch.float16, 128),
    ("EPI_BIAS", 4000, 256, 1024, torch.float16, 64),
    ("EPI_BIAS_WSILU", 32640, 256, 512, torch.float16, 0),
    ("EPI_BIAS_RES", 8160, 512, 256, torch.float16, 0),
    ("EPI_BIAS_RES_Q", 3000, 512, 256, torch.float16, 0),
    ("EPI_BIAS_RES2", 3000, 256, 256, torch.float16, 0),
    ("EPI_QUAD", 32640, 1024, 512, torch.float16, 0),
    ("EPI_QUAD", 2040, 1024, 256, torch.float16, 0),
    ("EPI_QUAD", 8160, 3072, 768, torch.float16, 0),
    ("EPI_BIAS_RES", 700, 192, 256, torch.float16, 64),
    ("EPI_BIAS_WSILU", 1300, 256, 128, torch.float16, 64),
    ("EPI_BIAS_RES_Q", 2000, 256, 512, torch.float16, 128),
    ("EPI_BIAS_RES2", 2100, 512, 512, torch.float16, 256),
    ("EPI_BIAS_Q", 1500, 512, 512, torch.float16, 0),
    ("EPI_BIAS", 5000, 512, 512, torch.bfloat16, 0),
    ("EPI_QUAD", 5000, 1024, 512, torch.bfloat16, 0),
    ("EPI_BIAS_RES", 5000, 512, 256, torch.bfloat16, 0),
]


@pytest.mark.parametrize("name,M,Nn,K,dtype,bn", CASES)
def test_conv1x1(name, M, Nn, K, dtype, bn):
    from dcvc_b200 import _native as N, ops
    epi = getattr(N, name)
    g = torch.Generator(device="cuda").manual_seed(M * 7 + Nn * 3 + K)
    dev = "cuda"
    # strided A (a channel slice of a wider buffer) to exercise the row pitch
    abuf = torch.randn(M, K + 64, device=dev, generator=g).to(dtype)
    a = abuf[:, 32:32 + K]
    w = (torch.randn(Nn, K, device=dev, generator=g) / K ** 0.5).to(dtype)
    b = torch.randn(Nn, device=dev, generator=g) * 0.1
    res = torch.randn(M, Nn, device=dev, generator=g).to(dtype)
    res2 = torch.randn(M, Nn, device=dev, generator=g).to(dtype)
    q = (torch.rand(Nn, device=dev, generator=g) + 0.5).to(dtype)
    out = ops.conv1x1(a, w, b, epi, res=res, res2=res2, qscale=q, block_n=bn)
    torch.cuda.synchronize()
    assert N.device_error() == 0
    ref = _ref(epi, a, w, b, res, res2, q)
    atol, rtol = TOL[dtype]
    err = (out.float() - ref).abs()
    assert bool((err <= atol + rtol * ref.abs()).all()), float(err.max())


@pytest.mark.parametrize("H,W,Cin,Cout", [(17, 30, 128, 256), (34, 60, 256, 256), (68, 120, 256, 512)])
def test_subpel(H, W, Cin, Cout):
    from dcvc_b200 import _native as N, ops
    g = torch.Generator(device="cuda").manual_seed(H * W)
    x = torch.randn(H * W, Cin, device="cuda", generator=g).half()
    w = (torch.randn(4 * Cout, Cin, device="cuda", generator=g) / Cin ** 0.5).half()
    out = ops.conv1x1(x, w, None, N.EPI_SUBPEL, sub_w=W, sub_cout=Cout)
    torch.cuda.synchronize()
    ref = _ref(N.EPI_SUBPEL, x, w, None, sub_w=W, sub_cout=Cout)
    err = (out.float() - ref).abs()
    assert bool((err <= 2e-2 + 1e-2 * ref.abs()).all()), float(err.max())


STREAM_CASES = [
    # (epilogue name, M, N, K, dtype): dc.3 / ffn.2 at 1080p, y-level shapes, ragged and tiny M
    ("EPI_BIAS_RES", 32640, 512, 256, torch.float16),
    ("EPI_BIAS_RES", 8160, 256, 256, torch.float16),
    ("EPI_BIAS_RES", 8160, 768, 192, torch.float16),
    ("EPI_BIAS_RES_Q", 32640, 512, 256, torch.float16),
    ("EPI_BIAS_RES", 4471, 384, 128, torch.float16),
    ("EPI_BIAS_RES", 37, 128, 64, torch.float16),
    ("EPI_BIAS_RES", 32640, 512, 256, torch.bfloat16),
    ("EPI_BIAS_RES_Q", 3000, 256, 256, torch.bfloat16),
    # bias / WSiLU epilogues at K <= 512: dc.0 at 1080p and at the y level, ragged shapes
    ("EPI_BIAS_WSILU", 32640, 256, 512, torch.float16),
    ("EPI_BIAS_WSILU", 8160, 256, 512, torch.bfloat16),
    ("EPI_BIAS_WSILU", 2047, 640, 448, torch.float16),
    ("EPI_BIAS", 4471, 384, 320, torch.float16),
    ("EPI_BIAS", 37, 128, 64, torch.bfloat16),
]


@pytest.mark.parametrize("name,M,Nn,K,dtype", STREAM_CASES)
def test_stream_form_matches_tiled_bitwise(name, M, Nn, K, dtype):
    """The streaming GEMM (W slice resident, row ranges per CTA) gives bitwise the tiled kernel's
    outputs for the residual, bias and WSiLU epilogues, and both are within the fp32-reference
    tolerance."""
    from dcvc_b200 import _native as N, ops
    epi = getattr(N, name)
    g = torch.Generator(device="cuda").manual_seed(M + Nn + K)
    abuf = torch.randn(M, K + 64, device="cuda", generator=g).to(dtype)
    a = abuf[:, 64:64 + K]
    w = (torch.randn(Nn, K, device="cuda", generator=g) / K ** 0.5).to(dtype)
    b = torch.randn(Nn, device="cuda", generator=g) * 0.1
    rbuf = torch.randn(M, Nn + 128, device="cuda", generator=g).to(dtype)
    res = rbuf[:, 128:]
    q = (torch.rand(Nn, device="cuda", generator=g) + 0.5).to(dtype)
    tiled = ops.conv1x1(a, w, b, epi, res=res, qscale=q, block_n=128 if Nn % 256 else 256)
    obuf = torch.full((M, Nn + 64), 7.0, device="cuda", dtype=dtype)
    stream = ops.conv1x1(a, w, b, epi, res=res, qscale=q, out=obuf[:, 64:], block_n=N.BLOCK_N_STREAM)
    torch.cuda.synchronize()
    assert N.device_error() == 0
    assert torch.equal(stream.view(torch.int16), tiled.view(torch.int16))
    assert bool((obuf[:, :64] == 7.0).all())  # nothing written outside the output view
    ref = _ref(epi, a, w, b, res, None, q)
    atol, rtol = TOL[dtype]
    assert bool(((stream.float() - ref).abs() <= atol + rtol * ref.abs()).all())


def test_quantize_fp8_matches_torch_cast():
    from dcvc_b200 import ops
    g = torch.Generator(device="cuda").manual_seed(5)
    for dtype in (torch.float16, torch.bfloat16):
        xb = (torch.randn(777, 320, device="cuda", generator=g) * 3).to(dtype)
        x = xb[:, 64:]
        q = ops.quantize_fp8(x, 1.0 / 0.75)
        ref = (x.float() * (1.0 / 0.75)).to(torch.float8_e4m3fn)
        assert torch.equal(q.view(torch.uint8), ref.view(torch.uint8))
    big = torch.full((8, 8), 6.0e4, device="cuda", dtype=torch.float16)
    assert float(ops.quantize_fp8(big, 1.0).float().max()) == 448.0  # saturates


@pytest.mark.parametrize("name,M,Nn,K,bn", [("EPI_QUAD", 32640, 1024, 512, 256),
                                             ("EPI_QUAD", 3000, 1024, 256, 256),
                                             ("EPI_BIAS_WSILU", 5000, 256, 512, 128),
                                             ("EPI_BIAS", 2047, 512, 384, 256)])
def test_conv1x1_f8_matches_dequantised_fp32(name, M, Nn, K, bn):
    """E4M3 operands with per-output-channel scales (kind::f8f6f4, FP32 accumulation) against
    an fp32 GEMM of the same dequantised operands; BF16 output tolerance."""
    from dcvc_b200 import _native as N, ops
    epi = getattr(N, name)
    g = torch.Generator(device="cuda").manual_seed(M + K)
    x = torch.randn(M, K, device="cuda", generator=g).to(torch.bfloat16)
    w = torch.randn(Nn, K, device="cuda", generator=g) / K ** 0.5
    b = torch.randn(Nn, device="cuda", generator=g) * 0.1
    a_scale = 0.5
    w_scale = w.abs().amax(1) / 448.0
    wq = (w / w_scale[:, None]).to(torch.float8_e4m3fn)
    aq = ops.quantize_fp8(x, 1.0 / a_scale)
    out = ops.conv1x1_f8(aq, wq, (w_scale * a_scale).float().contiguous(), b, epi, block_n=bn)
    torch.cuda.synchronize()
    assert N.device_error() == 0
    ad = aq.float() * a_scale
    wd = wq.float() * w_scale[:, None]
    ref = _ref(epi, ad, wd, b)
    err = (out.float() - ref).abs()
    assert bool((err <= 6e-2 + 2e-2 * ref.abs()).all()), float(err.max())


@pytest.mark.parametrize("form", ["tiled", "stream"])
def test_bounded_wait_runs_out_and_the_gpu_keeps_answering(form):
    """A GEMM whose producer issues no loads (injected) must give up on its waits after the short
    limit, report DCVC_DEVICE_TIMEOUT through the error word, and leave the context usable: the
    same GEMM right after it gives the right result.  No trap, no fault, no hang."""
    import ctypes
    from dcvc_b200 import _native as N, ops
    lib = N.lib
    lib.dcvc_gemm_inject_stall.argtypes = [ctypes.c_int, ctypes.c_longlong]
    lib.dcvc_check_device_errors.argtypes = [ctypes.c_void_p]
    g = torch.Generator(device="cuda").manual_seed(9)
    M, Nn, K = 4096, 512, 256
    a = torch.randn(M, K, device="cuda", generator=g).half()
    w = (torch.randn(Nn, K, device="cuda", generator=g) / K ** 0.5).half()
    b = torch.randn(Nn, device="cuda", generator=g) * 0.1
    res = torch.randn(M, Nn, device="cuda", generator=g).half()
    epi, bn = (N.EPI_BIAS, 256) if form == "tiled" else (N.EPI_BIAS_RES, N.BLOCK_N_STREAM)
    stream = torch.cuda.current_stream().cuda_stream
    assert lib.dcvc_check_device_errors(stream) == 0
    assert lib.dcvc_gemm_inject_stall(1, 20000) == 0  # ~10 us at 2 GHz
    ops.conv1x1(a, w, b, epi, res=res, block_n=bn)
    assert lib.dcvc_check_device_errors(stream) == 3  # DCVC_DEVICE_TIMEOUT
    assert b"bounded wait" in lib.dcvc_last_error()
    out = ops.conv1x1(a, w, b, epi, res=res, block_n=bn)
    assert lib.dcvc_check_device_errors(stream) == 0
    ref = _ref(epi, a, w, b, res)
    assert bool(((out.float() - ref).abs() <= 2e-2 + 1e-2 * ref.abs()).all())


DW_CASES = [
    # (H, W, img_h, K, N, dtype): dc.3 of a 512-channel block at 1080p; y-level; stacked images
    # with an odd width; a grid narrower than one warp's 16 pixels; one-row images
    (136, 240, 0, 256, 512, torch.float16),
    (136, 240, 0, 256, 512, torch.bfloat16),
    (68, 120, 0, 256, 256, torch.float16),
    (26, 52, 13, 256, 128, torch.float16),
    (26, 52, 13, 128, 384, torch.bfloat16),
    (5, 7, 0, 64, 128, torch.float16),
    (3, 300, 1, 192, 256, torch.float16),
]


@pytest.mark.parametrize("H,W,img_h,K,Nn,dtype", DW_CASES)
def test_depthwise_form_is_bitwise_the_two_launches(H, W, img_h, K, Nn, dtype):
    """The depthwise form of the streaming residual GEMM (the depthwise 3x3 computed by its operand
    producer) gives bitwise the outputs of the depthwise kernel followed by the residual GEMM, and
    is within tolerance of an fp32 torch reference of the two steps."""
    from dcvc_b200 import _native as N, ops
    M = H * W
    g = torch.Generator(device="cuda").manual_seed(H * W + K)
    xbuf = torch.randn(M, K + 64, device="cuda", generator=g).to(dtype)
    x = xbuf[:, 64:]
    dw = torch.randn(9, K, device="cuda", generator=g) * 0.3
    w = (torch.randn(Nn, K, device="cuda", generator=g) / K ** 0.5).to(dtype)
    b = torch.randn(Nn, device="cuda", generator=g) * 0.1
    res = torch.randn(M, Nn, device="cuda", generator=g).to(dtype)
    t = ops.dwconv3x3_ex(x, H, W, dw, img_h=img_h)
    split = ops.conv1x1(t, w, b, N.EPI_BIAS_RES, res=res, block_n=N.BLOCK_N_STREAM)
    tiled = ops.conv1x1(t, w, b, N.EPI_BIAS_RES, res=res, block_n=128)
    obuf = torch.full((M, Nn + 64), 7.0, device="cuda", dtype=dtype)
    fused = ops.dw3x3_conv1x1_res(x, H, W, dw, w, b, res, img_h=img_h, out=obuf[:, 64:])
    torch.cuda.synchronize()
    assert N.device_error() == 0
    assert torch.equal(fused.view(torch.int16), split.view(torch.int16))
    assert torch.equal(fused.view(torch.int16), tiled.view(torch.int16))
    assert bool((obuf[:, :64] == 7.0).all())
    # fp32 reference: per-image zero-padded depthwise conv, rounded to the activation type
    ih = img_h if img_h > 0 else H
    xi = x.float().reshape(H // ih, ih, W, K).permute(0, 3, 1, 2)
    d = torch.nn.functional.conv2d(xi, dw.t().reshape(K, 1, 3, 3), padding=1, groups=K)
    d = d.permute(0, 2, 3, 1).reshape(M, K).to(dtype).float()
    ref = d @ w.float().t() + b + res.float()
    atol, rtol = TOL[dtype]
    assert bool(((fused.float() - ref).abs() <= atol + rtol * ref.abs()).all())


def test_depthwise_form_bounded_wait_runs_out():
    """The depthwise form's producers skip their work under the stall injection; the MMA and
    epilogue waits run out, the launch reports DCVC_DEVICE_TIMEOUT and the next launch is right."""
    import ctypes
    from dcvc_b200 import _native as N, ops
    lib = N.lib
    lib.dcvc_gemm_inject_stall.argtypes = [ctypes.c_int, ctypes.c_longlong]
    lib.dcvc_check_device_errors.argtypes = [ctypes.c_void_p]
    g = torch.Generator(device="cuda").manual_seed(13)
    H, W, K, Nn = 32, 64, 256, 512
    x = torch.randn(H * W, K, device="cuda", generator=g).half()
    dw = torch.randn(9, K, device="cuda", generator=g) * 0.3
    w = (torch.randn(Nn, K, device="cuda", generator=g) / K ** 0.5).half()
    b = torch.randn(Nn, device="cuda", generator=g) * 0.1
    res = torch.randn(H * W, Nn, device="cuda", generator=g).half()
    stream = torch.cuda.current_stream().cuda_stream
    assert lib.dcvc_check_device_errors(stream) == 0
    assert lib.dcvc_gemm_inject_stall(1, 20000) == 0
    ops.dw3x3_conv1x1_res(x, H, W, dw, w, b, res)
    assert lib.dcvc_check_device_errors(stream) == 3  # DCVC_DEVICE_TIMEOUT
    out = ops.dw3x3_conv1x1_res(x, H, W, dw, w, b, res)
    assert lib.dcvc_check_device_errors(stream) == 0
    t = ops.dwconv3x3_ex(x, H, W, dw)
    ref = ops.conv1x1(t, w, b, N.EPI_BIAS_RES, res=res, block_n=N.BLOCK_N_STREAM)
    assert torch.equal(out.view(torch.int16), ref.view(torch.int16))


PAIR_CASES = [
    # (epilogue name, M, N, K, dtype): the quad GEMM at 1080p and at a ragged M (the last 256-row
    # tile half empty), dc.0 at the y level, a small bias GEMM, BF16
    ("EPI_QUAD", 32640, 1024, 512, torch.float16),
    ("EPI_QUAD", 3000, 1024, 256, torch.float16),
    ("EPI_BIAS_WSILU", 8160, 256, 512, torch.float16),
    ("EPI_BIAS", 777, 512, 128, torch.float16),
    ("EPI_QUAD", 8160, 1024, 512, torch.bfloat16),
]


@pytest.mark.parametrize("name,M,Nn,K,dtype", PAIR_CASES)
def test_pair_form_matches_tiled(name, M, Nn, K, dtype):
    """The CTA-pair form (cta_group::2: 256 x 256 tiles over two SMs, each staging half of W)
    against the one-SM tiled kernel and the fp32 reference.  The products are summed in the same
    K order; whether the tensor cores round M = 256 tiles exactly as M = 128 tiles is printed."""
    from dcvc_b200 import _native as N, ops
    epi = getattr(N, name)
    g = torch.Generator(device="cuda").manual_seed(M + Nn + K + 1)
    a = torch.randn(M, K, device="cuda", generator=g).to(dtype)
    w = (torch.randn(Nn, K, device="cuda", generator=g) / K ** 0.5).to(dtype)
    b = torch.randn(Nn, device="cuda", generator=g) * 0.1
    nout = Nn // 4 if epi == N.EPI_QUAD else Nn
    tiled = ops.conv1x1(a, w, b, epi, block_n=256)
    obuf = torch.full((M, nout + 64), 7.0, device="cuda", dtype=dtype)
    pair = ops.conv1x1(a, w, b, epi, out=obuf[:, 64:], block_n=N.BLOCK_N_PAIR)
    torch.cuda.synchronize()
    assert N.device_error() == 0
    assert bool((obuf[:, :64] == 7.0).all())
    same = torch.equal(pair.view(torch.int16), tiled.view(torch.int16))
    print(f"pair form {name} {M}x{Nn}x{K} {dtype}: bitwise equal to the tiled kernel: {same}, "
          f"max |diff| {float((pair.float() - tiled.float()).abs().max()):.3e}")
    ref = _ref(epi, a, w, b)
    atol, rtol = TOL[dtype]
    assert bool(((pair.float() - ref).abs() <= atol + rtol * ref.abs()).all())


def test_pair_form_bounded_wait_runs_out():
    """Under the stall injection neither CTA of a pair loads anything: the even CTA's MMA wait and
    the odd CTA's epilogue wait run out, the launch reports DCVC_DEVICE_TIMEOUT, both CTAs meet at
    the final cluster barrier, and the next launch is right."""
    import ctypes
    from dcvc_b200 import _native as N, ops
    lib = N.lib
    lib.dcvc_gemm_inject_stall.argtypes = [ctypes.c_int, ctypes.c_longlong]
    lib.dcvc_check_device_errors.argtypes = [ctypes.c_void_p]
    g = torch.Generator(device="cuda").manual_seed(21)
    M, Nn, K = 4096, 1024, 256
    a = torch.randn(M, K, device="cuda", generator=g).half()
    w = (torch.randn(Nn, K, device="cuda", generator=g) / K ** 0.5).half()
    b = torch.randn(Nn, device="cuda", generator=g) * 0.1
    stream = torch.cuda.current_stream().cuda_stream
    assert lib.dcvc_check_device_errors(stream) == 0
    assert lib.dcvc_gemm_inject_stall(1, 20000) == 0
    ops.conv1x1(a, w, b, N.EPI_QUAD, block_n=N.BLOCK_N_PAIR)
    assert lib.dcvc_check_device_errors(stream) == 3  # DCVC_DEVICE_TIMEOUT
    out = ops.conv1x1(a, w, b, N.EPI_QUAD, block_n=N.BLOCK_N_PAIR)
    assert lib.dcvc_check_device_errors(stream) == 0
    ref = _ref(N.EPI_QUAD, a, w, b)
    assert bool(((out.float() - ref).abs() <= 2e-2 + 1e-2 * ref.abs()).all())
