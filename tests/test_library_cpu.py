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


def test_compaction_entry_points_reject_bad_pointers_without_gpu():
    """Null or misaligned pointers are refused on the host with DCVC_INVALID_ARGUMENT before any
    CUDA call, so a ctypes caller gets a status instead of a device memory fault (no GPU here:
    a launch would fail with a CUDA error, status 2, not 1)."""
    from dcvc_b200 import _native as N
    vp, i = ctypes.c_void_p, ctypes.c_int
    f = N.lib.dcvc_compact
    f.restype, f.argtypes = i, [vp, i, vp, i, vp, vp, vp, vp]
    g = N.lib.dcvc_compact_noalloc
    g.restype, g.argtypes = i, [vp, i, vp, i, vp, vp, vp]
    r = N.lib.dcvc_recover
    r.restype, r.argtypes = i, [vp, vp, vp, i, vp, vp]
    ok = 0x10000  # an aligned stand-in address; never dereferenced because a check fails first
    cases = [
        (None, 2, ok, ok, ok, ok),      # null src
        (ok, 2, None, ok, ok, ok),      # null cond
        (ok, 2, ok, ok, None, ok),      # null dst
        (ok, 2, ok, ok, ok, None),      # null total
        (ok, 2, ok + 4, ok, ok, ok),    # cond not 8-byte aligned
        (ok + 1, 2, ok, ok, ok, ok),    # 2-byte src misaligned
        (ok, 2, ok, ok, ok + 1, ok),    # 2-byte dst misaligned
        (ok, 2, ok, ok, ok, ok + 2),    # total misaligned
        (ok, 3, ok, ok, ok, ok),        # element size
    ]
    for src, eb, cond, counts, dst, total in cases:
        assert f(src, eb, cond, 1000, counts, dst, total, None) == 1, (src, eb, cond, dst, total)
        assert b"alignment" in N.lib.dcvc_last_error()
        assert g(src, eb, cond, 1000, dst, total, None) == 1, (src, eb, cond, dst, total)
    assert f(ok, 2, ok, 1000, None, ok, ok, None) == 1        # null block counts
    assert f(ok, 2, ok, 0, ok, ok, ok, None) == 1             # empty input
    assert r(ok, ok, None, 1000, ok, None) == 1               # recover: null block counts
    assert r(ok, ok, ok, 1000, ok + 1, None) == 1             # recover: misaligned FP16 output
    assert r(None, ok, ok, 1000, ok, None) == 1               # recover: null decoded values
