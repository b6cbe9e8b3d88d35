"""The reference models' own call sequence into inference_extensions_cuda, replayed on the GPU.

tests/golden/dropin_calls.json records every call the unmodified reference DMC (HT-S) and DMCI
models made into the drop-in proxies (made by tests/golden/make_dropin_golden.py from the
reference sources; they cannot be imported where this test runs).  Here the same sequence runs
on the real proxies: a fresh proxy per model instance as the reference creates them, set_param
with the seeded state dict whose entries equal the recorded ones (checked on the CPU by
tests/test_dropin_calls_cpu.py), then add_ref_feature_from_frame / compress / decompress with the
recorded arguments (tensors of the recorded shape, dtype and memory format, filled with
synthetic content; the payload of each compress feeds the matching decompress).  The results
must have the shapes and types the reference models consume, and the decoder must reproduce the
encoder: the intra reconstruction exactly, the video codec's entropy parameters, symbols and
y_hat bit for bit after each chunk."""
import json
import os

import numpy as np
import pytest
import torch

from dcvc_b200.entropy_tables import add_cdf_to_state_dict
from dcvc_b200.model_spec import perturbed_dmci_state_dict, perturbed_hts_state_dict

pytestmark = pytest.mark.gpu


def _tensor(desc, seed):
    g = torch.Generator().manual_seed(seed)
    t = (torch.rand(*desc["tensor"], generator=g) - 0.5).to(getattr(torch, desc["dtype"])).cuda()
    return t.contiguous(memory_format=torch.channels_last) if desc["channels_last"] else t


def test_reference_call_sequence_replays_on_the_proxies():
    from dcvc_b200.inference_extensions_cuda import DMCHTSProxy, DMCIProxy
    log = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "dropin_calls.json")))
    hp = (log["height"] + 15) // 16 * 16
    wp = (log["width"] + 15) // 16 * 16
    sds = {"DMC": perturbed_hts_state_dict, "DMCI": perturbed_dmci_state_dict}
    classes = {"DMC": DMCHTSProxy, "DMCI": DMCIProxy}
    seeds = {("DMC", "add_ref_feature_from_frame"): 7, ("DMC", "compress"): 11,
             ("DMCI", "compress"): 13}
    proxy, payloads, intra_hat, enc_state = {}, {"DMC": [], "DMCI": []}, [], []
    for c in log["calls"]:
        m = c["model"]
        if c["call"] == "__init__":
            proxy[m] = classes[m]()
            continue
        p = proxy[m]
        if c["call"] == "set_param":
            sd = add_cdf_to_state_dict(sds[m](0))
            sd = {k: (v.half().cuda() if v.is_floating_point() else v) for k, v in sd.items()}
            p.set_param(sd, c["skip_threshold"])
            continue
        args = []
        for a in c["args"]:
            if "tensor" in a:
                args.append(_tensor(a, seeds[(m, c["call"])]))
            elif "array" in a:
                args.append(payloads[m].pop(0))  # the matching compress's payload
            else:
                args.append(a["value"])
        out = getattr(p, c["call"])(*args)
        torch.cuda.synchronize()
        if c["call"] == "compress":
            bits = out[0]
            assert isinstance(bits, np.ndarray) and bits.dtype == np.uint8 and bits.size > 0
            payloads[m].append(bits)
            if m == "DMCI":
                intra_hat.append(out[1].clone())
            else:
                enc_state.append({n: p.buffer(n).clone() for n in ("common", "y_q", "y_hat")})
        elif c["call"] == "decompress":
            if m == "DMCI":
                assert out.shape == (1, 3, hp, wp) and out.dtype == torch.float16
                assert torch.equal(out, intra_hat.pop(0))  # the encoder's reconstruction
            else:
                assert isinstance(out, list) and len(out) == 8
                assert all(f.shape == (1, 3, hp, wp) and f.dtype == torch.float16 for f in out)
                for n, t in enc_state.pop(0).items():
                    assert torch.equal(p.buffer(n).view(torch.int16), t.view(torch.int16)), n
    assert not payloads["DMC"] and not payloads["DMCI"] and not enc_state and not intra_hat
