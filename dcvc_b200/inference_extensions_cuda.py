"""Drop-in for the reference's `inference_extensions_cuda` module (src/layers/extensions/
inference/bind.cpp:11-39): the same proxy classes, methods, argument meaning and return values,
backed by the sm_100a runtime in libdcvc_b200.so.

DMCHTSProxy and DMCHTLProxy (the HT-S and HT-L chunk codecs), DMCLDProxy (the low-delay frame
codec) and DMCIProxy (the intra model) are all implemented.
"""
import ctypes

import numpy as np
import torch

from . import _native as N

_lib = N.lib
_vp = ctypes.c_void_p


def _proto(name, argtypes):
    f = getattr(_lib, name)
    f.restype = ctypes.c_int
    f.argtypes = argtypes
    return f


for _k in ("hts", "htl", "ld"):
    _proto(f"dcvc_{_k}_create", [ctypes.POINTER(_vp)])
    _proto(f"dcvc_{_k}_destroy", [_vp])
    _proto(f"dcvc_{_k}_set_param", [_vp, ctypes.c_int, ctypes.POINTER(ctypes.c_char_p),
                                     ctypes.POINTER(_vp), ctypes.POINTER(ctypes.c_int64),
                                     ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                     ctypes.POINTER(ctypes.c_int), ctypes.c_float])
    _proto(f"dcvc_{_k}_add_ref_feature", [_vp, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp])
    _proto(f"dcvc_{_k}_compress", [_vp, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                    ctypes.c_int, ctypes.c_int, _vp, ctypes.POINTER(_vp),
                                    ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_int)])
    _proto(f"dcvc_{_k}_decompress", [_vp, _vp, ctypes.c_size_t, ctypes.c_int, ctypes.c_int,
                                      ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp,
                                      ctypes.POINTER(_vp)])
    _proto(f"dcvc_{_k}_buffer", [_vp, ctypes.c_char_p, ctypes.POINTER(_vp), ctypes.POINTER(ctypes.c_int),
                                  ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)])
    _proto(f"dcvc_{_k}_stats", [_vp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                 ctypes.POINTER(ctypes.c_size_t)])
_proto("dcvc_hts_set_precision", [_vp, ctypes.c_int])
_proto("dcvc_hts_share_params", [_vp, _vp])
_proto("dcvc_hts_add_ref_features", [_vp, ctypes.POINTER(_vp), ctypes.c_int, ctypes.c_int,
                                     ctypes.c_int, ctypes.c_int, _vp])
_proto("dcvc_hts_compress_batch", [_vp, ctypes.POINTER(_vp), ctypes.c_int, ctypes.c_int,
                                   ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.c_int,
                                   ctypes.c_int, ctypes.c_int, _vp,
                                   ctypes.POINTER(ctypes.POINTER(_vp)),
                                   ctypes.POINTER(ctypes.POINTER(ctypes.c_size_t)),
                                   ctypes.POINTER(ctypes.c_int)])
_proto("dcvc_hts_decompress_batch", [_vp, ctypes.POINTER(_vp), ctypes.POINTER(ctypes.c_size_t),
                                     ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                     ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp,
                                     ctypes.POINTER(_vp)])
_proto("dcvc_hts_state_bytes", [_vp, ctypes.POINTER(ctypes.c_size_t)])
_proto("dcvc_hts_export_state", [_vp, _vp, _vp, ctypes.POINTER(ctypes.c_int)])
_proto("dcvc_hts_import_state", [_vp, _vp, ctypes.c_int, _vp])
_proto("dcvc_hts_buffer_dtype", [_vp, ctypes.c_char_p, ctypes.POINTER(ctypes.c_int)])
_proto("dcvc_hts_set_timing", [_vp, ctypes.c_int])
_proto("dcvc_hts_recon_branches", [ctypes.c_int])
_proto("dcvc_hts_timing", [_vp, ctypes.POINTER(ctypes.c_float), ctypes.c_int, ctypes.POINTER(ctypes.c_int)])
_proto("dcvc_intra_create", [ctypes.POINTER(_vp)])
_proto("dcvc_intra_destroy", [_vp])
_proto("dcvc_intra_set_param", [_vp, ctypes.c_int, ctypes.POINTER(ctypes.c_char_p),
                                ctypes.POINTER(_vp), ctypes.POINTER(ctypes.c_int64),
                                ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                ctypes.POINTER(ctypes.c_int), ctypes.c_float])
_proto("dcvc_intra_compress", [_vp, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                               ctypes.c_int, _vp, ctypes.POINTER(_vp),
                               ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_int),
                               ctypes.POINTER(_vp)])
_proto("dcvc_intra_decompress", [_vp, _vp, ctypes.c_size_t, ctypes.c_int, ctypes.c_int,
                                 ctypes.c_int, ctypes.c_int, _vp, ctypes.POINTER(_vp)])
_proto("dcvc_intra_buffer", [_vp, ctypes.c_char_p, ctypes.POINTER(_vp), ctypes.POINTER(ctypes.c_int),
                             ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)])
_proto("dcvc_intra_stats", [_vp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                            ctypes.POINTER(ctypes.c_size_t)])

_DTYPES = {torch.float16: 0, torch.bfloat16: 1, torch.float32: 2, torch.int32: 3, torch.int64: 4}
FRAMES = 8


class _DeviceView:
    """__cuda_array_interface__ over memory owned by the native runtime (no copy)."""

    def __init__(self, ptr, shape, typestr="<f2"):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": typestr,
                                         "data": (int(ptr), False), "version": 3, "strides": None}


def _stream():
    return _vp(torch.cuda.current_stream().cuda_stream)


def _channels_last_data(t, name):
    if not t.is_cuda or t.dtype != torch.float16 or t.dim() != 4 or t.shape[0] != 1:
        raise ValueError(f"{name} must be a [1, C, H, W] float16 CUDA tensor")
    if not t.is_contiguous(memory_format=torch.channels_last):
        t = t.contiguous(memory_format=torch.channels_last)
    return t


def _bytes_out(data, size):
    if size.value == 0:
        return np.zeros(0, dtype=np.uint8)
    return np.ctypeslib.as_array(ctypes.cast(data, ctypes.POINTER(ctypes.c_uint8)),
                                 shape=(size.value,)).copy()


class _Proxy:
    """Handle lifetime, set_param, buffer and stats shared by the codec proxies; `_kind` selects
    the dcvc_<kind>_* entry points."""

    _kind = ""

    def __init__(self):
        h = _vp()
        N.check(self._fn("create")(ctypes.byref(h)), f"{type(self).__name__}()")
        self._h = h

    def _fn(self, name):
        return getattr(_lib, f"dcvc_{self._kind}_{name}")

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            self._fn("destroy")(h)
            self._h = None

    def set_param(self, state_dict, skip_threshold):
        """state_dict: the model state dict with the four CDF entries added
        (common_model.py:64-70); tensors may be on any device, in f16/bf16/f32/int."""
        keep = []
        names, ptrs, shapes, ndims, dtypes, on_dev = [], [], [], [], [], []
        for k, v in state_dict.items():
            if not isinstance(v, torch.Tensor):
                v = torch.as_tensor(np.asarray(v))
            if v.dtype not in _DTYPES:
                v = v.float()
            v = v.contiguous()
            keep.append(v)
            names.append(k.encode())
            ptrs.append(v.data_ptr())
            shp = list(v.shape)[:4] + [0] * (4 - min(4, v.dim()))
            if v.dim() > 4:
                raise ValueError(f"state-dict entry {k} has more than 4 dimensions")
            shapes.extend(shp)
            ndims.append(v.dim())
            dtypes.append(_DTYPES[v.dtype])
            on_dev.append(1 if v.is_cuda else 0)
        n = len(names)
        if any(v.is_cuda for v in keep):
            torch.cuda.current_stream().synchronize()
        N.check(self._fn("set_param")(
            self._h, n, (ctypes.c_char_p * n)(*names), (_vp * n)(*ptrs),
            (ctypes.c_int64 * (4 * n))(*shapes), (ctypes.c_int * n)(*ndims),
            (ctypes.c_int * n)(*dtypes), (ctypes.c_int * n)(*on_dev), float(skip_threshold)),
            "set_param")

    def _buffer_dtype(self, name):
        return torch.float16

    def buffer(self, name):
        """Copy of an internal device buffer as a [rows, cols] float16 (or, in the HT-S codec's
        BF16 form, bfloat16) tensor (see dcvc_hts_buffer / dcvc_intra_buffer)."""
        ptr, r, c, ld = _vp(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        N.check(self._fn("buffer")(self._h, name.encode(), ctypes.byref(ptr), ctypes.byref(r),
                                   ctypes.byref(c), ctypes.byref(ld)), "buffer")
        full = torch.as_tensor(_DeviceView(ptr.value, (r.value, ld.value), "<i2"), device="cuda")
        torch.cuda.synchronize()
        return full[:, : c.value].clone().view(self._buffer_dtype(name))

    def stats(self):
        """(symbols coded by the last call, kernels it enqueued, device bytes held)."""
        s, k, b = ctypes.c_int(), ctypes.c_int(), ctypes.c_size_t()
        N.check(self._fn("stats")(self._h, ctypes.byref(s), ctypes.byref(k), ctypes.byref(b)),
                "stats")
        return s.value, k.value, b.value


class DMCHTSProxy(_Proxy):
    """Chunk codec of the HT-S video model (dmc_hts_proxy.h:215-355).  One instance per stream;
    not re-entrant.

    precision: "fp16" (the reference's form, default), "bf16" — the activation format of the
    analysis and synthesis transforms — or "fp8" (the BF16 form with the transforms' quad GEMMs
    on E4M3 operands), see dcvc_hts_set_precision; an extension, the reference's constructor
    takes no arguments.  Inputs and reconstructions stay float16 in every form."""

    _kind = "hts"
    _PRECISIONS = {"fp16": 0, "bf16": 1, "fp8": 2}

    def __init__(self, precision="fp16"):
        super().__init__()
        if precision not in self._PRECISIONS:
            raise ValueError(f"precision must be one of {sorted(self._PRECISIONS)}")
        if self._kind == "hts":
            N.check(_lib.dcvc_hts_set_precision(self._h, self._PRECISIONS[precision]),
                    "set_precision")
        elif precision != "fp16":
            raise ValueError(f"{type(self).__name__} runs in the fp16 form only")
        self.precision = precision

    # ---- packed batches: n streams of one resolution per call (HT-S only; an extension)
    TIMING_NAMES = ("enc_analysis", "enc_update", "enc_update_reset", "dec_temporal",
                    "dec_temporal_memory", "dec_hyper", "dec_context", "dec_synthesis",
                    "host_wait_analysis", "host_rans_encode", "host_decode_z", "host_wait_hyper",
                    "host_decode_y")

    def set_timing(self, enable=True):
        """Times the phase graphs (CUDA events) and the host's waits and entropy coding of the
        following calls; timing() returns the last call's values in milliseconds."""
        N.check(_lib.dcvc_hts_set_timing(self._h, 1 if enable else 0), "set_timing")

    def timing(self):
        """{name: ms} for the parts the last compress / decompress ran."""
        out = (ctypes.c_float * len(self.TIMING_NAMES))()
        n = ctypes.c_int()
        N.check(_lib.dcvc_hts_timing(self._h, out, len(out), ctypes.byref(n)), "timing")
        return {k: round(float(out[i]), 4) for i, k in enumerate(self.TIMING_NAMES[:n.value])
                if out[i] >= 0}

    def add_ref_features_from_frames(self, frames, apply_adaptor=True):
        """Seeds n streams (and sizes the codec for them) from n [1, 3, Hp, Wp] float16 frames."""
        self._hts_only("add_ref_features_from_frames")
        frames = [_channels_last_data(f, "frame") for f in frames]
        n = len(frames)
        ptrs = (_vp * n)(*[f.data_ptr() for f in frames])
        N.check(_lib.dcvc_hts_add_ref_features(self._h, ptrs, n, frames[0].shape[2],
                                               frames[0].shape[3], 1 if apply_adaptor else 0,
                                               _stream()), "add_ref_features_from_frames")

    def compress_batch(self, xs, qps, reset_feature_memory, padding_b, padding_r):
        """xs: n [1, 24, H, W] float16 CUDA chunks, qps: n QPs.  Returns n (uint8 array,
        ec_parallel) pairs, each equal to what a single-stream proxy returns for that stream."""
        self._hts_only("compress_batch")
        xs = [_channels_last_data(x, "x") for x in xs]
        n = len(xs)
        ptrs = (_vp * n)(*[x.data_ptr() for x in xs])
        q = (ctypes.c_int * n)(*[int(v) for v in qps])
        data = ctypes.POINTER(_vp)()
        sizes = ctypes.POINTER(ctypes.c_size_t)()
        ecp = (ctypes.c_int * n)()
        N.check(_lib.dcvc_hts_compress_batch(self._h, ptrs, n, xs[0].shape[2], xs[0].shape[3], q,
                                             1 if reset_feature_memory else 0, int(padding_b),
                                             int(padding_r), _stream(), ctypes.byref(data),
                                             ctypes.byref(sizes), ecp), "compress_batch")
        out = []
        for k in range(n):
            sz = ctypes.c_size_t(sizes[k])
            out.append((_bytes_out(_vp(data[k]), sz), ecp[k]))
        return out

    def decompress_batch(self, payloads, qps, height, width, ec_parallels, reset_feature_memory):
        """n payloads -> 8 [n, 3, Hp, Wp] float16 CUDA tensors (frame i of every stream; stream k
        is index k), aliasing the proxy's buffers until its next call."""
        self._hts_only("decompress_batch")
        bs = [np.ascontiguousarray(np.asarray(b, dtype=np.uint8).reshape(-1)) for b in payloads]
        n = len(bs)
        ptrs = (_vp * n)(*[b.ctypes.data for b in bs])
        sizes = (ctypes.c_size_t * n)(*[b.size for b in bs])
        q = (ctypes.c_int * n)(*[int(v) for v in qps])
        e = (ctypes.c_int * n)(*[int(v) for v in ec_parallels])
        frames = (_vp * FRAMES)()
        N.check(_lib.dcvc_hts_decompress_batch(self._h, ptrs, sizes, q, e, n, int(height),
                                               int(width), 1 if reset_feature_memory else 0,
                                               _stream(), frames), "decompress_batch")
        hp = (int(height) + 15) // 16 * 16
        wp = (int(width) + 15) // 16 * 16
        return [torch.as_tensor(_DeviceView(frames[i], (n, hp, wp, 3)), device="cuda").permute(0, 3, 1, 2)
                for i in range(FRAMES)]

    # ---- extensions for serving many streams (HT-S only; no counterpart in the reference)
    def share_params_from(self, other):
        """Use `other`'s prepared parameters (same device) instead of a set_param of our own."""
        self._hts_only("share_params_from")
        N.check(_lib.dcvc_hts_share_params(self._h, other._h), "share_params_from")
        self.precision = other.precision

    def state_bytes(self):
        self._hts_only("state_bytes")
        n = ctypes.c_size_t()
        N.check(_lib.dcvc_hts_state_bytes(self._h, ctypes.byref(n)), "state_bytes")
        return n.value

    def export_state(self, out=None):
        """The stream's temporal context as (uint8 CUDA tensor, flags), copied on the current
        stream (into `out` when given)."""
        self._hts_only("export_state")
        n = self.state_bytes()
        if out is None:
            out = torch.empty(n, dtype=torch.uint8, device="cuda")
        if out.numel() < n or not out.is_cuda:
            raise ValueError(f"state buffer must be a CUDA uint8 tensor of {n} bytes")
        flags = ctypes.c_int()
        N.check(_lib.dcvc_hts_export_state(self._h, out.data_ptr(), _stream(), ctypes.byref(flags)),
                "export_state")
        return out, flags.value

    def import_state(self, state, flags):
        """Replaces the temporal context with one exported at the same resolution and form."""
        self._hts_only("import_state")
        if state.numel() < self.state_bytes():
            raise ValueError("state buffer is smaller than this codec's state")
        N.check(_lib.dcvc_hts_import_state(self._h, state.data_ptr(), int(flags), _stream()),
                "import_state")

    def _hts_only(self, what):
        if self._kind != "hts":
            raise NotImplementedError(f"{what} is implemented for DMCHTSProxy only")

    def _buffer_dtype(self, name):
        if self._kind != "hts":
            return torch.float16
        dt = ctypes.c_int()
        N.check(_lib.dcvc_hts_buffer_dtype(self._h, name.encode(), ctypes.byref(dt)), "buffer")
        return torch.bfloat16 if dt.value == 1 else torch.float16

    def add_ref_feature_from_frame(self, frame, apply_adaptor=True):
        frame = _channels_last_data(frame, "frame")
        if frame.shape[1] != 3:
            raise ValueError("frame must have 3 channels")
        N.check(self._fn("add_ref_feature")(self._h, frame.data_ptr(), frame.shape[2],
                                            frame.shape[3], 1 if apply_adaptor else 0,
                                            _stream()), "add_ref_feature_from_frame")

    def compress(self, x, qp, reset_feature_memory, padding_b, padding_r):
        """x: [1, 24, H, W] float16 CUDA (8 frames).  Returns (uint8 array, ec_parallel)."""
        x = _channels_last_data(x, "x")
        data = _vp()
        size = ctypes.c_size_t()
        ecp = ctypes.c_int()
        N.check(self._fn("compress")(self._h, x.data_ptr(), x.shape[2], x.shape[3], int(qp),
                                     1 if reset_feature_memory else 0, int(padding_b),
                                     int(padding_r), _stream(), ctypes.byref(data),
                                     ctypes.byref(size), ctypes.byref(ecp)), "compress")
        return _bytes_out(data, size), ecp.value

    def decompress(self, bit_stream, qp, height, width, entropy_coder_parallel,
                   reset_feature_memory):
        """Returns 8 [1, 3, Hp, Wp] float16 CUDA tensors (channels last) that alias the proxy's
        buffers and are overwritten by the next call (dmc_hts_proxy.h:347)."""
        bs = np.ascontiguousarray(np.asarray(bit_stream, dtype=np.uint8).reshape(-1))
        frames = (_vp * FRAMES)()
        N.check(self._fn("decompress")(self._h, bs.ctypes.data, bs.size, int(qp), int(height),
                                       int(width), int(entropy_coder_parallel),
                                       1 if reset_feature_memory else 0, _stream(), frames),
                "decompress")
        hp = (int(height) + 15) // 16 * 16
        wp = (int(width) + 15) // 16 * 16
        out = []
        for i in range(FRAMES):
            t = torch.as_tensor(_DeviceView(frames[i], (1, hp, wp, 3)), device="cuda")
            out.append(t.permute(0, 3, 1, 2))
        return out



class DMCHTLProxy(DMCHTSProxy):
    """Chunk codec of the HT-L video model (dmc_htl_proxy.h): the DMCHTSProxy interface, with
    4-step entropy coding inside (bind.cpp:19-24)."""

    _kind = "htl"


class DMCIProxy(_Proxy):
    """Intra (DMCI) frame codec (dmci_proxy.h:132-230).  Not re-entrant."""

    _kind = "intra"

    def compress(self, x, qp, padding_b, padding_r):
        """x: [1, 3, H, W] float16 CUDA.  Returns (uint8 array, x_hat, ec_parallel), x_hat a
        [1, 3, H + padding_b, W + padding_r] float16 CUDA tensor (channels last) aliasing the
        proxy's buffer (overwritten by the next call)."""
        x = _channels_last_data(x, "x")
        if x.shape[1] != 3:
            raise ValueError("x must have 3 channels")
        data, size, ecp, xh = _vp(), ctypes.c_size_t(), ctypes.c_int(), _vp()
        N.check(_lib.dcvc_intra_compress(self._h, x.data_ptr(), x.shape[2], x.shape[3], int(qp),
                                         int(padding_b), int(padding_r), _stream(),
                                         ctypes.byref(data), ctypes.byref(size),
                                         ctypes.byref(ecp), ctypes.byref(xh)), "compress")
        hp, wp = x.shape[2] + int(padding_b), x.shape[3] + int(padding_r)
        x_hat = torch.as_tensor(_DeviceView(xh.value, (1, hp, wp, 3)), device="cuda")
        return _bytes_out(data, size), x_hat.permute(0, 3, 1, 2), ecp.value

    def decompress(self, bit_stream, qp, height, width, entropy_coder_parallel):
        """Returns the [1, 3, Hp, Wp] float16 reconstruction (Hp, Wp = height, width rounded up
        to multiples of 16), aliasing the proxy's buffer."""
        bs = np.ascontiguousarray(np.asarray(bit_stream, dtype=np.uint8).reshape(-1))
        xh = _vp()
        N.check(_lib.dcvc_intra_decompress(self._h, bs.ctypes.data, bs.size, int(qp), int(height),
                                           int(width), int(entropy_coder_parallel), _stream(),
                                           ctypes.byref(xh)), "decompress")
        hp = (int(height) + 15) // 16 * 16
        wp = (int(width) + 15) // 16 * 16
        x_hat = torch.as_tensor(_DeviceView(xh.value, (1, hp, wp, 3)), device="cuda")
        return x_hat.permute(0, 3, 1, 2)


class DMCLDProxy(DMCHTSProxy):
    """Low-delay frame codec (dmc_ld_proxy.h, bind.cpp:33-38): the DMCHTSProxy interface on one
    frame per call.  Not re-entrant."""

    _kind = "ld"

    def compress(self, x, qp, reset_feature_memory, padding_b, padding_r):
        """x: [1, 3, H, W] float16 CUDA.  Returns (uint8 array, ec_parallel)."""
        if x.dim() != 4 or x.shape[1] != 3:
            raise ValueError("x must be a [1, 3, H, W] tensor")
        return super().compress(x, qp, reset_feature_memory, padding_b, padding_r)

    def decompress(self, bit_stream, qp, height, width, entropy_coder_parallel,
                   reset_feature_memory):
        """Returns the [1, 3, Hp, Wp] float16 reconstruction (channels last), aliasing the
        proxy's buffer (overwritten by the next call)."""
        bs = np.ascontiguousarray(np.asarray(bit_stream, dtype=np.uint8).reshape(-1))
        xh = _vp()
        N.check(self._fn("decompress")(self._h, bs.ctypes.data, bs.size, int(qp), int(height),
                                       int(width), int(entropy_coder_parallel),
                                       1 if reset_feature_memory else 0, _stream(), ctypes.byref(xh)),
                "decompress")
        hp = (int(height) + 15) // 16 * 16
        wp = (int(width) + 15) // 16 * 16
        x_hat = torch.as_tensor(_DeviceView(xh.value, (1, hp, wp, 3)), device="cuda")
        return x_hat.permute(0, 3, 1, 2)
