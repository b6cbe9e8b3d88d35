"""Records how the reference's own models call the drop-in modules (tests/golden/dropin_calls.json).

Run here, where the reference checkout exists (--ref or DCVC_REFERENCE):

    python tests/golden/make_dropin_golden.py [--ref <reference checkout>]

The unmodified reference models `DMC(ModelStructure.HTS)` (src/models/video_model_ht.py) and
`DMCI()` (src/models/image_model.py) are built under torch.manual_seed(0), `update(0.15)`, and
driven through their public inference calls (add_ref_feature_from_frame, compress, decompress)
with `dcvc_b200.dropin.install()` in place.  The proxy classes they import are replaced by
recorders that check every call against the signature of dcvc_b200's proxy method it stands for
and log the call: the state dict passed to set_param (name, shape, dtype of every entry) and, for
the other methods, each argument's kind (tensor shape / dtype / memory format, array dtype, or
the plain value).  No GPU is needed: the recorders return outputs of the documented shapes.
The GPU test tests/test_dropin_replay_gpu.py replays the log on the real proxies.
"""
import argparse
import inspect
import json
import os
import sys

import numpy as np
import torch

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
OUT = os.path.join(ROOT, "tests", "golden", "dropin_calls.json")


def describe(v):
    if isinstance(v, torch.Tensor):
        cl = v.dim() == 4 and v.is_contiguous(memory_format=torch.channels_last)
        return {"tensor": list(v.shape), "dtype": str(v.dtype).replace("torch.", ""),
                "channels_last": bool(cl)}
    if isinstance(v, np.ndarray):
        return {"array": list(v.shape), "dtype": str(v.dtype)}
    if isinstance(v, (bool, int, float, str)) or v is None:
        return {"value": v}
    return {"type": type(v).__name__}


def make_recorder(real_cls, log, model):
    frames = 8

    class Recorder:
        def __init__(self, *a, **k):
            inspect.signature(real_cls.__init__).bind(self, *a, **k)
            log.append({"model": model, "call": "__init__", "args": [describe(x) for x in a]})

        def _rec(self, name, a, k):
            inspect.signature(getattr(real_cls, name)).bind(self, *a, **k)
            log.append({"model": model, "call": name, "args": [describe(x) for x in a],
                        "kwargs": {kk: describe(vv) for kk, vv in k.items()}})

        def set_param(self, state_dict, skip_threshold):
            inspect.signature(real_cls.set_param).bind(self, state_dict, skip_threshold)
            log.append({"model": model, "call": "set_param",
                        "state_dict": [[n, list(t.shape), str(t.dtype).replace("torch.", "")]
                                       for n, t in state_dict.items()],
                        "skip_threshold": float(skip_threshold)})

        def add_ref_feature_from_frame(self, *a, **k):
            self._rec("add_ref_feature_from_frame", a, k)

        def compress(self, *a, **k):
            self._rec("compress", a, k)
            data = np.zeros(16, dtype=np.uint8)
            if model == "DMCI":
                x = a[0]
                hp, wp = x.shape[2] + a[2], x.shape[3] + a[3]
                return data, torch.zeros(1, 3, hp, wp, dtype=x.dtype), 1
            return data, 1

        def decompress(self, *a, **k):
            self._rec("decompress", a, k)
            h, w = a[2], a[3]
            hp, wp = (h + 15) // 16 * 16, (w + 15) // 16 * 16
            if model == "DMCI":
                return torch.zeros(1, 3, hp, wp, dtype=torch.float16)
            return [torch.zeros(1, 3, hp, wp, dtype=torch.float16) for _ in range(frames)]

    return Recorder


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("DCVC_REFERENCE"),
                    help="reference checkout (default: $DCVC_REFERENCE)")
    args = ap.parse_args()
    if not args.ref:
        ap.error("give --ref or set DCVC_REFERENCE to the reference checkout")
    sys.path.insert(0, ROOT)
    sys.path.insert(0, args.ref)
    from dcvc_b200 import dropin, inference_extensions_cuda as iec
    from src.models.image_model import DMCI
    from src.models.video_model_ht import DMC
    from src.utils.common import ModelStructure

    log = []
    dropin.install()
    real = {"DMCHTSProxy": iec.DMCHTSProxy, "DMCIProxy": iec.DMCIProxy}
    iec.DMCHTSProxy = make_recorder(real["DMCHTSProxy"], log, "DMC")
    iec.DMCIProxy = make_recorder(real["DMCIProxy"], log, "DMCI")
    try:
        H, W = 200, 248
        pad_b, pad_r = (-H) % 16, (-W) % 16
        torch.manual_seed(0)
        intra = DMCI()
        intra.update(0.15)
        intra = intra.half().eval()
        x1 = torch.zeros(1, 3, H, W, dtype=torch.float16).contiguous(memory_format=torch.channels_last)
        with torch.no_grad():
            enc = intra.compress(x1, 32, pad_b, pad_r)
            intra.decompress(enc["bit_stream"], {"height": H, "width": W}, 32, enc["ec_parallel"])
        torch.manual_seed(0)
        video = DMC(ModelStructure.HTS)
        video.update(0.15)
        video = video.half().eval()
        ref = torch.zeros(1, 3, H + pad_b, W + pad_r, dtype=torch.float16)
        ref = ref.contiguous(memory_format=torch.channels_last)
        x = torch.zeros(1, 24, H, W, dtype=torch.float16).contiguous(memory_format=torch.channels_last)
        with torch.no_grad():
            video.add_ref_feature_from_frame(ref, True)
            for qp, reset in ((21, False), (42, True)):
                out = video.compress(x, qp, reset, pad_b, pad_r)
            video.proxy = None  # a decoder is a model instance of its own in the reference harness
            video.add_ref_feature_from_frame(ref, False)
            for qp, reset in ((21, False), (42, True)):
                video.decompress(out["bit_stream"], {"height": H, "width": W}, qp,
                                 out["ec_parallel"], reset)
    finally:
        iec.DMCHTSProxy, iec.DMCIProxy = real["DMCHTSProxy"], real["DMCIProxy"]
        dropin.uninstall()
    with open(OUT, "w") as f:
        json.dump({"height": H, "width": W, "calls": log}, f, indent=0)
    print(f"wrote {OUT}: {len(log)} calls")


if __name__ == "__main__":
    main()
