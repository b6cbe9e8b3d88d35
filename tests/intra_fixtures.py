"""Shared helpers for the intra (DMCI) codec tests: seeded model state and synthetic frames."""
import functools

from dcvc_b200 import synthetic
from dcvc_b200.entropy_tables import add_cdf_to_state_dict
from dcvc_b200.model_spec import dmci_state_dict, perturbed_dmci_state_dict

SKIP_THRES = 0.15


@functools.lru_cache(maxsize=4)
def intra_state_dict(seed=0, perturbed=True, device="cuda"):
    """fp16 intra state dict with CDF tables; perturbed=True: calibrated weights with per-QP
    quant vectors, False: the exact random init."""
    sd = perturbed_dmci_state_dict(seed) if perturbed else dmci_state_dict(seed)
    sd = add_cdf_to_state_dict(sd)
    return {k: (v.half().to(device) if v.is_floating_point() else v) for k, v in sd.items()}


def make_intra_proxy(sd):
    from dcvc_b200.inference_extensions_cuda import DMCIProxy
    p = DMCIProxy()
    p.set_param(sd, SKIP_THRES)
    return p


def intra_frame(H, W, seed=1, device="cuda"):
    """(model input [1, 3, H, W] float16 channels-last, (y, u, v) uint8 planes)."""
    yuv = synthetic.intra_frame_yuv420(seed, H, W)
    return synthetic.to_model_input([yuv], device=device), yuv
