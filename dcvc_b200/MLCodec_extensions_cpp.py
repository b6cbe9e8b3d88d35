"""Drop-in for the reference's `MLCodec_extensions_cpp` module (src/cpp/py_rans/bind.cpp:14-40).

Same class and method names, argument meaning and byte format, backed by the C++ coder in
libdcvc_b200.so.  Two additions: `RansDecoder.get_decoded_tensor()` returns the symbols decoded
by the last decode_y / decode_z call (the reference only exposes them to C++,
py_rans.h:64), and errors raise RuntimeError instead of terminating a worker thread.
"""
import ctypes

import numpy as np

from . import _native as N

_lib = N.lib
_i32p = ctypes.POINTER(ctypes.c_int32)


def _proto(name, argtypes):
    f = getattr(_lib, name)
    f.restype = ctypes.c_int
    f.argtypes = argtypes
    return f


_proto("dcvc_pmf_to_quantized_cdf", [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p])
_proto("dcvc_ec_parallel_for", [ctypes.c_int])
_proto("dcvc_rans_create", [ctypes.POINTER(ctypes.c_void_p)])
_proto("dcvc_rans_destroy", [ctypes.c_void_p])
_proto("dcvc_rans_set_cdf", [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                             ctypes.c_int, ctypes.c_int])
_proto("dcvc_rans_encode_begin", [ctypes.c_void_p, ctypes.c_int])
_proto("dcvc_rans_encode_y", [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int])
_proto("dcvc_rans_encode_z", [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                              ctypes.c_int])
_proto("dcvc_rans_encode_finish", [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p),
                                   ctypes.POINTER(ctypes.c_size_t)])
_proto("dcvc_rans_decode_begin", [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int])
_proto("dcvc_rans_decode_z", [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                              ctypes.c_void_p])
_proto("dcvc_rans_decode_y", [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p])
_proto("dcvc_rans_inject_task_fault", [ctypes.c_int])


def pmf_to_quantized_cdf(pmf):
    """pmf (sequence of floats) -> list of len(pmf) + 1 cumulative frequencies summing to 2**16."""
    p = np.ascontiguousarray(np.asarray(pmf, dtype=np.float32))
    out = np.zeros(p.size + 1, dtype=np.uint32)
    N.check(_lib.dcvc_pmf_to_quantized_cdf(p.ctypes.data, p.size, out.ctypes.data),
            "pmf_to_quantized_cdf")
    return out.tolist()


def ec_parallel_for(symbol_count):
    return _lib.dcvc_ec_parallel_for(int(symbol_count))


def inject_task_fault(sub_stream):
    """Failure-path testing: the next coder task of `sub_stream` throws in its worker; the call
    raises DcvcError (DCVC_INTERNAL) and the coder stays usable.  -1 cancels."""
    N.check(_lib.dcvc_rans_inject_task_fault(int(sub_stream)), "inject_task_fault")


class _Coder:
    def __init__(self):
        h = ctypes.c_void_p()
        N.check(_lib.dcvc_rans_create(ctypes.byref(h)), "dcvc_rans_create")
        self._h = h
        self._ecp = 1

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            _lib.dcvc_rans_destroy(h)
            self._h = None

    def set_cdf(self, cdfs, cdfs_sizes, index):
        sizes = np.ascontiguousarray(np.asarray(cdfs_sizes, dtype=np.int32).reshape(-1))
        cdf = np.ascontiguousarray(np.asarray(cdfs, dtype=np.int32)).reshape(sizes.size, -1)
        N.check(_lib.dcvc_rans_set_cdf(self._h, int(index), cdf.ctypes.data, sizes.ctypes.data,
                                       sizes.size, cdf.shape[1]), "set_cdf")

    def set_entropy_coder_parallel(self, n):
        if not 1 <= int(n) <= 8:
            raise ValueError("entropy coder parallelism must be in [1, 8]")
        self._ecp = int(n)


class RansEncoder(_Coder):
    """Encoder: reset(), encode_y / encode_z in coding order, flush(), get_encoded_stream()."""

    def __init__(self):
        super().__init__()
        self._segments = []
        self._stream = np.zeros(0, dtype=np.uint8)

    def reset(self):
        self._segments = []

    def encode_y(self, symbols):
        self._segments.append(("y", np.ascontiguousarray(np.asarray(symbols, dtype=np.int16)
                                                         .reshape(-1))))

    def encode_z(self, symbols, cdf_offset, ch):
        self._segments.append(("z", np.ascontiguousarray(np.asarray(symbols, dtype=np.int8)
                                                         .reshape(-1)), int(cdf_offset), int(ch)))

    def flush(self):
        N.check(_lib.dcvc_rans_encode_begin(self._h, self._ecp), "encode")
        for seg in self._segments:
            if seg[0] == "y":
                N.check(_lib.dcvc_rans_encode_y(self._h, seg[1].ctypes.data, seg[1].size), "encode_y")
            else:
                N.check(_lib.dcvc_rans_encode_z(self._h, seg[1].ctypes.data, seg[1].size, seg[2],
                                                seg[3]), "encode_z")
        data = ctypes.c_void_p()
        size = ctypes.c_size_t()
        N.check(_lib.dcvc_rans_encode_finish(self._h, ctypes.byref(data), ctypes.byref(size)),
                "flush")
        self._stream = np.ctypeslib.as_array(
            ctypes.cast(data, ctypes.POINTER(ctypes.c_uint8)), shape=(size.value,)).copy() \
            if size.value else np.zeros(0, dtype=np.uint8)
        self._segments = []

    def get_encoded_stream(self):
        return self._stream


class RansDecoder(_Coder):
    """Decoder: set_stream(bytes), then decode_z / decode_y in the reverse order of encoding."""

    def __init__(self):
        super().__init__()
        self._decoded = np.zeros(0, dtype=np.int8)
        self._data = None

    def set_stream(self, encoded):
        self._data = np.ascontiguousarray(np.asarray(encoded, dtype=np.uint8).reshape(-1))
        N.check(_lib.dcvc_rans_decode_begin(self._h, self._data.ctypes.data, self._data.size,
                                            self._ecp), "set_stream")

    def decode_z(self, total_size, cdf_offset, ch):
        out = np.zeros(int(total_size), dtype=np.int8)
        N.check(_lib.dcvc_rans_decode_z(self._h, out.size, int(cdf_offset), int(ch),
                                        out.ctypes.data), "decode_z")
        self._decoded = out

    def decode_y(self, indexes):
        idx = np.ascontiguousarray(np.asarray(indexes, dtype=np.uint8).reshape(-1))
        out = np.zeros(idx.size, dtype=np.int8)
        N.check(_lib.dcvc_rans_decode_y(self._h, idx.ctypes.data, idx.size, out.ctypes.data),
                "decode_y")
        self._decoded = out

    def get_decoded_tensor(self):
        return self._decoded
