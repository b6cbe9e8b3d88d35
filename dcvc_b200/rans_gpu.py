"""The MLCodec rANS coder on the GPU (dcvc_rans_gpu_* in libdcvc_b200.so): byte-identical payloads
with the host coder (MLCodec_extensions_cpp here, the reference's src/cpp/py_rans), symbols and
payloads in device memory, up to 64 payloads per launch.  The container fixes the parallelism at
one thread per sub-stream (at most 8 per payload), so a single payload codes slower than on the
CPU threads; batching independent streams is what the GPU form is for."""
import ctypes

import torch

from . import MLCodec_extensions_cpp as M
from . import _native as N

_vp, _i = ctypes.c_void_p, ctypes.c_int
MAX_JOBS = 64


class EncJob(ctypes.Structure):
    _fields_ = [("y", _vp), ("n_y", _i), ("z", _vp), ("n_z", _i), ("z_offset", _i),
                ("z_ch", _i), ("ecp", _i), ("scratch", _vp), ("out", _vp), ("out_cap", _i),
                ("out_size", _vp), ("status", _vp)]


class DecJob(ctypes.Structure):
    _fields_ = [("data", _vp), ("size", _i), ("ecp", _i), ("n_z", _i), ("z_offset", _i),
                ("z_ch", _i), ("z_out", _vp), ("y_idx", _vp), ("n_y", _i), ("y_out", _vp),
                ("status", _vp)]


def _sig(name, res, args):
    f = getattr(N.lib, name)
    f.restype = res
    f.argtypes = args


_sig("dcvc_rans_gpu_create", _i, [_vp, ctypes.POINTER(_vp)])
_sig("dcvc_rans_gpu_destroy", _i, [_vp])
_sig("dcvc_rans_gpu_scratch_bytes", ctypes.c_size_t, [_i, _i, _i])
_sig("dcvc_rans_gpu_encode", _i, [_vp, ctypes.POINTER(EncJob), _i, _vp])
_sig("dcvc_rans_gpu_decode", _i, [_vp, ctypes.POINTER(DecJob), _i, _vp])

STATUS = {0: "ok", 1: "table index out of range", 2: "buffer overflow",
          3: "inconsistent container header", 4: "truncated or corrupt sub-stream",
          5: "symbol with zero probability"}


def _ptr(t):
    return None if t is None or t.numel() == 0 else t.data_ptr()


class GpuRansCoder:
    """Device copy of a z (bit-estimator) and a y (Gaussian) CDF table set."""

    def __init__(self, z_cdf, z_len, y_cdf, y_len):
        self._host = M.RansEncoder()
        self._host.set_cdf(z_cdf, z_len, 0)
        self._host.set_cdf(y_cdf, y_len, 1)
        h = _vp()
        N.check(N.lib.dcvc_rans_gpu_create(self._host._h, ctypes.byref(h)), "dcvc_rans_gpu_create")
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            N.lib.dcvc_rans_gpu_destroy(h)
            self._h = None

    def encode(self, jobs, stream=None):
        """jobs: list of dicts with y (int16 CUDA, (value << 8) + table index), z (int8 CUDA),
        z_offset, z_ch and ecp.  Returns (list of uint8 CUDA payloads, list of statuses)."""
        if not 1 <= len(jobs) <= MAX_JOBS:
            raise ValueError("1..64 jobs per call")
        arr = (EncJob * len(jobs))()
        keep = []
        dev = jobs[0]["y"].device
        meta = torch.zeros(2 * len(jobs), dtype=torch.int32, device=dev)
        outs = []
        for i, j in enumerate(jobs):
            y, z = j["y"], j["z"]
            ny, nz = y.numel(), z.numel()
            scratch = torch.empty(max(1, N.lib.dcvc_rans_gpu_scratch_bytes(ny, nz, j["ecp"])),
                                  dtype=torch.uint8, device=dev)
            cap = 4 * (ny + nz) + 64
            out = torch.empty(cap, dtype=torch.uint8, device=dev)
            keep += [scratch]
            outs.append(out)
            arr[i] = EncJob(_ptr(y), ny, _ptr(z), nz, j.get("z_offset", 0), j.get("z_ch", 1),
                            j["ecp"], scratch.data_ptr(), out.data_ptr(), cap,
                            meta.data_ptr() + 8 * i, meta.data_ptr() + 8 * i + 4)
        s = stream if stream is not None else torch.cuda.current_stream()
        N.check(N.lib.dcvc_rans_gpu_encode(self._h, arr, len(jobs), _vp(s.cuda_stream)),
                "dcvc_rans_gpu_encode")
        m = meta.view(-1, 2).cpu()
        return [o[: int(m[i, 0])] for i, o in enumerate(outs)], [int(m[i, 1]) for i in range(len(jobs))]

    def decode(self, jobs, stream=None):
        """jobs: list of dicts with data (uint8 CUDA payload), ecp, n_z, z_offset, z_ch and y_idx
        (uint8 CUDA table index per y symbol).  Returns (list of (z, y) int8 CUDA tensors, list
        of statuses)."""
        if not 1 <= len(jobs) <= MAX_JOBS:
            raise ValueError("1..64 jobs per call")
        arr = (DecJob * len(jobs))()
        dev = jobs[0]["data"].device
        status = torch.zeros(len(jobs), dtype=torch.int32, device=dev)
        res = []
        for i, j in enumerate(jobs):
            zo = torch.empty(j["n_z"], dtype=torch.int8, device=dev)
            yi = j["y_idx"]
            yo = torch.empty(yi.numel(), dtype=torch.int8, device=dev)
            res.append((zo, yo))
            arr[i] = DecJob(_ptr(j["data"]), j["data"].numel(), j["ecp"], j["n_z"],
                            j.get("z_offset", 0), j.get("z_ch", 1), _ptr(zo), _ptr(yi),
                            yi.numel(), _ptr(yo), status.data_ptr() + 4 * i)
        s = stream if stream is not None else torch.cuda.current_stream()
        N.check(N.lib.dcvc_rans_gpu_decode(self._h, arr, len(jobs), _vp(s.cuda_stream)),
                "dcvc_rans_gpu_decode")
        return res, status.cpu().tolist()
