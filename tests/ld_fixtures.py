"""Shared helpers for the low-delay (LD) codec tests: seeded model state and the LD proxy."""
import functools

from dcvc_b200 import synthetic
from dcvc_b200.entropy_tables import add_cdf_to_state_dict
from dcvc_b200.model_spec import ld_state_dict, perturbed_ld_state_dict

SKIP_THRES = 0.15


@functools.lru_cache(maxsize=2)
def ld_state_dict16(seed=0, perturbed=True, device="cuda"):
    """fp16 LD state dict with CDF tables; perturbed=True: calibrated weights with per-QP quant
    vectors, False: the exact random init."""
    sd = perturbed_ld_state_dict(seed) if perturbed else ld_state_dict(seed)
    sd = add_cdf_to_state_dict(sd)
    return {k: (v.half().to(device) if v.is_floating_point() else v) for k, v in sd.items()}


def make_ld_proxy(sd):
    from dcvc_b200.inference_extensions_cuda import DMCLDProxy
    p = DMCLDProxy()
    p.set_param(sd, SKIP_THRES)
    return p


def ld_frames(H, W, n, seed=2):
    """n + 1 synthetic YUV 4:2:0 frames: the first seeds the reference, the rest are coded."""
    return synthetic.video_chunk_yuv420(seed, H, W, n + 1, 0)
