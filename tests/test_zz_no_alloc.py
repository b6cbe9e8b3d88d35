"""The allocation-free compaction entry point (dcvc_compact_noalloc), called through the C ABI.

It exists for callers that cannot allocate device memory themselves — for example a serving
process whose device memory is pre-partitioned by its own allocator, or a latency-critical path
that cannot take cudaMalloc's implicit synchronisation — and so cannot provide the per-call
block-count buffer that dcvc_compact needs.  Its scratch is a fixed array inside the library.
Two calls in a row (the second sees the first call's leftover scratch) must give exactly the
same result as dcvc_compact with a caller buffer and as the CPU oracle's compaction; sizes beyond
the built-in maximum are refused.  This file is collected last on purpose."""
import ctypes
import os
import sys

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

MAX_ELEMENTS = 4096 * 8192
sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import elementwise_oracle  # noqa: E402


def _lib():
    from dcvc_b200 import _native as N
    f = N.lib.dcvc_compact_noalloc
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                  ctypes.c_void_p, ctypes.c_void_p]
    return N


def _noalloc(src, cond):
    N = _lib()
    dst = torch.full_like(src, 0)
    total = torch.full((1,), -1, dtype=torch.int32, device=src.device)
    st = N.lib.dcvc_compact_noalloc(src.data_ptr(), src.element_size(), cond.data_ptr(), src.numel(),
                                    dst.data_ptr(), total.data_ptr(),
                                    torch.cuda.current_stream().cuda_stream)
    assert st == 0, N.lib.dcvc_last_error()
    return dst, total


def test_no_alloc_compaction_matches_compact_twice():
    from dcvc_b200 import ops
    rng = np.random.default_rng(123)
    # first call: the 1080p latent count; second call: a smaller, ragged size (its blocks reuse
    # the scratch the first call left behind)
    cases = [(2088960, np.int16, 0.15), (100003, np.uint8, 0.6)]
    for n, dtype, density in cases:
        cond = torch.from_numpy((rng.random(n) < density).astype(np.uint8)).cuda()
        if dtype == np.int16:
            src = torch.from_numpy(rng.integers(-32768, 32767, n).astype(np.int16)).cuda()
        else:
            src = torch.from_numpy(rng.integers(0, 256, n).astype(np.uint8)).cuda()
        ref_dst, ref_total, _ = ops.compact(src, cond)
        dst, total = _noalloc(src, cond)
        torch.cuda.synchronize()
        k = int(ref_total.item())
        assert int(total.item()) == k == int(cond.sum().item())
        assert torch.equal(dst[:k], ref_dst[:k])
        want, kw = elementwise_oracle.compact(src.cpu().numpy(), cond.cpu().numpy())
        assert kw == k and np.array_equal(dst[:k].cpu().numpy(), want)


def test_no_alloc_rejects_sizes_beyond_its_scratch():
    N = _lib()
    st = N.lib.dcvc_compact_noalloc(None, 1, None, MAX_ELEMENTS + 1, None, None, None)
    assert st == 1
    assert b"exceeds the maximum" in N.lib.dcvc_last_error()
