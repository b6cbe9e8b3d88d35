"""ctypes binding of libdcvc_b200.so (the C ABI declared in include/dcvc_b200.h).

The library is required: there is no CPU or PyTorch fallback for any operator of this package.
If it is missing, importing this module raises.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libdcvc_b200.so")

if not os.path.exists(LIB_PATH):
    raise ImportError(
        f"{LIB_PATH} is missing: build it with `python -m dcvc_b200.build` (nvcc, sm_100a)")

lib = ctypes.CDLL(LIB_PATH)

c_int = ctypes.c_int
c_vp = ctypes.c_void_p
c_float_p = ctypes.POINTER(ctypes.c_float)

# status codes (include/dcvc_b200.h)
DCVC_OK = 0
STATUS_NAMES = {
    1: "invalid argument", 2: "CUDA error", 3: "device timeout", 4: "out of memory",
    5: "corrupt stream", 6: "not ready", 7: "host timeout", 8: "internal error",
}

F16, BF16 = 0, 1
EPI_BIAS, EPI_BIAS_WSILU, EPI_BIAS_RES, EPI_BIAS_RES_Q, EPI_BIAS_RES2, EPI_QUAD, EPI_SUBPEL, \
    EPI_BIAS_Q = range(8)
BLOCK_N_STREAM = -1  # dcvc_conv1x1 block_n: the streaming form of the residual epilogues
BLOCK_N_PAIR = -2  # dcvc_conv1x1 block_n: the CTA-pair form (cta_group::2) of bias / WSiLU / quad


class DcvcError(RuntimeError):
    """Raised when a C-ABI call returns a non-zero status."""

    def __init__(self, status, where):
        msg = lib.dcvc_last_error().decode(errors="replace")
        super().__init__(f"{where}: {STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


def check(status, where):
    if status != DCVC_OK:
        raise DcvcError(status, where)


def _proto(name, restype, argtypes):
    f = getattr(lib, name)
    f.restype = restype
    f.argtypes = argtypes
    return f


_proto("dcvc_last_error", ctypes.c_char_p, [])
_proto("dcvc_abi_version", c_int, [])
_proto("dcvc_device_error", c_int, [ctypes.POINTER(c_int), c_int])
_proto("dcvc_conv1x1", c_int,
       [c_int, c_int, c_int, c_int, c_int, c_vp, c_int, c_vp, c_vp, c_vp, c_int, c_vp, c_int,
        c_vp, c_vp, c_int, c_int, c_int, c_int, c_vp])


_proto("dcvc_gemm_autotune", c_int, [c_int, c_int, c_int, c_int, c_int, c_int, c_int, c_vp,
                                    ctypes.POINTER(c_int), ctypes.POINTER(ctypes.c_float)])
_proto("dcvc_gemm_autotune_enable", c_int, [c_int])
_proto("dcvc_gemm_tuned", c_int, [c_int, c_int, c_int, c_int, c_int, c_int, ctypes.POINTER(c_int)])
_proto("dcvc_gemm_tuning_clear", c_int, [])
_proto("dcvc_conv_ffn", c_int, [c_int, c_int, c_int, c_vp, c_int, c_vp, c_vp, c_vp, c_vp, c_vp,
                               c_vp, c_int, c_int, c_vp])
_proto("dcvc_dwconv3x3", c_int, [c_vp, c_int, c_int, c_int, c_int, c_vp, c_vp, c_int, c_vp])
_proto("dcvc_dwconv3x3_ex", c_int, [c_int, c_vp, c_int, c_int, c_int, c_int, c_int, c_vp, c_vp, c_int, c_vp])
_proto("dcvc_dw3x3_conv1x1_res", c_int, [c_int, c_int, c_int, c_int, c_vp, c_int, c_vp, c_int, c_vp, c_int,
                                        c_vp, c_vp, c_int, c_vp, c_int, c_vp])
_proto("dcvc_dw_fusion", c_int, [c_int])
_proto("dcvc_gemm_pair_form", c_int, [c_int])
_proto("dcvc_hts_recon_branches", c_int, [c_int])


def device_error(clear=True):
    code = c_int(0)
    check(lib.dcvc_device_error(ctypes.byref(code), 1 if clear else 0), "dcvc_device_error")
    return code.value
