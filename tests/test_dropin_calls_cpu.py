"""The calls the unmodified reference models make into the drop-in modules, checked on the CPU
against this package's proxies (no GPU and no reference sources needed: the calls were recorded
from the reference by tests/golden/make_dropin_golden.py)."""
import inspect
import json
import os

import pytest


def test_recorded_reference_calls_fit_the_dropin_proxies():
    """Every recorded call binds to the drop-in proxy method it targets, and the state dicts the
    reference passes to set_param are, entry for entry (name, shape, dtype), the ones this
    package's seeded model specs produce, so set_param sees exactly the keys the codecs were
    built for."""
    from dcvc_b200.entropy_tables import add_cdf_to_state_dict
    from dcvc_b200.inference_extensions_cuda import DMCHTSProxy, DMCIProxy
    from dcvc_b200.model_spec import dmci_state_dict, hts_state_dict
    log = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "dropin_calls.json")))
    classes = {"DMC": DMCHTSProxy, "DMCI": DMCIProxy}
    specs = {"DMC": hts_state_dict, "DMCI": dmci_state_dict}
    seen = set()
    for c in log["calls"]:
        cls = classes[c["model"]]
        seen.add((c["model"], c["call"]))
        if c["call"] == "set_param":
            sd = add_cdf_to_state_dict(specs[c["model"]](0))
            mine = {k: [list(v.shape), str((v.half() if v.is_floating_point() else v).dtype)[6:]]
                    for k, v in sd.items()}
            ref = {n: [s, t] for n, s, t in c["state_dict"]}
            assert mine == ref, c["model"]
            assert c["skip_threshold"] == pytest.approx(0.15)
            continue
        args = [None] * len(c.get("args", []))
        inspect.signature(getattr(cls, c["call"])).bind(None, *args, **c.get("kwargs", {}))
    assert {("DMC", "compress"), ("DMC", "decompress"), ("DMC", "add_ref_feature_from_frame"),
            ("DMCI", "compress"), ("DMCI", "decompress")} <= seen
