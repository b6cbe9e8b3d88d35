"""Shared helpers for the HT-L codec tests: seeded model state and the HT-L proxy."""
import functools

from dcvc_b200.entropy_tables import add_cdf_to_state_dict
from dcvc_b200.model_spec import htl_state_dict, perturbed_htl_state_dict

SKIP_THRES = 0.15


@functools.lru_cache(maxsize=2)
def htl_state_dict16(seed=0, perturbed=True, device="cuda"):
    """fp16 HT-L state dict with CDF tables; perturbed=True: calibrated weights with per-QP
    quant vectors, False: the exact random init."""
    sd = perturbed_htl_state_dict(seed) if perturbed else htl_state_dict(seed)
    sd = add_cdf_to_state_dict(sd)
    return {k: (v.half().to(device) if v.is_floating_point() else v) for k, v in sd.items()}


def make_htl_proxy(sd):
    from dcvc_b200.inference_extensions_cuda import DMCHTLProxy
    p = DMCHTLProxy()
    p.set_param(sd, SKIP_THRES)
    return p
