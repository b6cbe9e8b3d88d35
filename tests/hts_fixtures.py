"""Shared helpers for the HT-S codec tests: seeded model state and synthetic chunks."""
import functools

from dcvc_b200 import synthetic
from dcvc_b200.entropy_tables import add_cdf_to_state_dict
from dcvc_b200.model_spec import hts_state_dict, perturbed_hts_state_dict

SKIP_THRES = 0.15


@functools.lru_cache(maxsize=4)
def state_dict(seed=0, perturbed=True, device="cuda"):
    """fp16 state dict with CDF tables (built from the fp32 parameters first, as the reference
    harness runs update() before .half()).  perturbed=True: the calibrated seed-0 weights with
    per-QP quant vectors (numerically stable); False: the exact random init."""
    sd = perturbed_hts_state_dict(seed) if perturbed else hts_state_dict(seed)
    sd = add_cdf_to_state_dict(sd)
    out = {}
    for k, v in sd.items():
        out[k] = v.half().to(device) if v.is_floating_point() else v
    return out


def make_proxy(sd):
    from dcvc_b200.inference_extensions_cuda import DMCHTSProxy
    p = DMCHTSProxy()
    p.set_param(sd, SKIP_THRES)
    return p


def chunk(H, W, start, seed=2):
    return synthetic.to_model_input(synthetic.video_chunk_yuv420(seed, H, W, 8, start))


def ref_frame(H, W, seed=2):
    f = synthetic.video_chunk_yuv420(seed, H, W, 1, 0)[0]
    return synthetic.padded_reference_frame(f)
