"""The C-ABI library loads on a machine without a GPU and exports every function that
include/dcvc_b200.h declares; host-only entry points work."""
import ctypes
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    text = open(os.path.join(ROOT, "include", "dcvc_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(dcvc_[a-z0-9_]+)\s*\(", text)))


def test_every_declared_symbol_is_exported():
    from dcvc_b200 import _native as N
    names = declared_functions()
    assert len(names) >= 40
    missing = [n for n in names if not hasattr(N.lib, n)]
    assert not missing, missing


def test_host_entry_points_without_gpu():
    from dcvc_b200 import _native as N
    assert N.lib.dcvc_abi_version() == 1
    lut = (ctypes.c_uint8 * 65536)()
    N.lib.dcvc_scale_index_table.argtypes = [ctypes.c_void_p]
    assert N.lib.dcvc_scale_index_table(lut) == 0
    assert lut[0x3C00] == 56  # scale 1.0 -> floor((0 + 2.207) * 25.5) = 56
    N.lib.dcvc_conv1x1.restype = ctypes.c_int
    # invalid dtype is rejected before any device work
    st = N.lib.dcvc_conv1x1(9, 0, 128, 128, 64, None, 64, None, None, None, 0, None, 0, None,
                            None, 128, 0, 0, 0, None)
    assert st == 1 and b"dtype" in N.lib.dcvc_last_error()


def test_tuner_and_fault_hook_entry_points_without_gpu():
    """The autotuner's host entry points answer without a GPU (an empty table, a status for the
    tuning call itself), and the coder's fault hook accepts and cancels an injection."""
    from dcvc_b200 import _native as N
    from dcvc_b200 import MLCodec_extensions_cpp as M  # noqa: F401  (binds the fault hook)
    bn = ctypes.c_int(-1)
    assert N.lib.dcvc_gemm_tuning_clear() == 0
    assert N.lib.dcvc_gemm_tuned(0, N.EPI_BIAS, 1000, 256, 512, 0, ctypes.byref(bn)) == 0
    assert bn.value == 0
    assert N.lib.dcvc_gemm_tuned(0, N.EPI_BIAS, 1000, 256, 512, 0, None) == 1  # null output
    assert N.lib.dcvc_gemm_autotune(9, N.EPI_BIAS, 1000, 256, 512, 0, 0, None, None, None) == 1
    # without a device the tuning call fails with a status (no crash, nothing recorded)
    st = N.lib.dcvc_gemm_autotune(0, N.EPI_BIAS, 1000, 256, 512, 0, 0, None, ctypes.byref(bn), None)
    assert st != 0
    assert N.lib.dcvc_gemm_tuned(0, N.EPI_BIAS, 1000, 256, 512, 0, ctypes.byref(bn)) == 0
    assert bn.value == 0
    assert N.lib.dcvc_gemm_autotune_enable(0) == 0
    assert N.lib.dcvc_rans_inject_task_fault(2) == 0
    assert N.lib.dcvc_rans_inject_task_fault(-1) == 0
