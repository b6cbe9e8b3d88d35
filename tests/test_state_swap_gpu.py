"""A stream's temporal context outside the codec: export it from one codec and import it into
another that shares the first one's parameters, and the second codec codes the stream's next
chunk to the same bytes and reconstruction as the first would have (encoder and decoder side)."""
import numpy as np
import pytest
import torch

from dcvc_b200 import synthetic
from tests.hts_fixtures import chunk, ref_frame, state_dict

pytestmark = pytest.mark.gpu


def test_exported_state_continues_on_another_codec():
    from dcvc_b200.inference_extensions_cuda import DMCHTSProxy
    sd = state_dict()
    H, W = 200, 248
    pr, pb = synthetic.padding_for(H, W)
    a_enc, a_dec = DMCHTSProxy(), DMCHTSProxy()
    a_enc.set_param(sd, 0.15)
    a_dec.set_param(sd, 0.15)
    b_enc, b_dec = DMCHTSProxy(), DMCHTSProxy()
    b_enc.share_params_from(a_enc)
    b_dec.share_params_from(a_enc)
    ref = ref_frame(H, W)
    a_enc.add_ref_feature_from_frame(ref, True)
    a_dec.add_ref_feature_from_frame(ref, False)
    b_enc.add_ref_feature_from_frame(ref_frame(H, W, seed=9), True)   # other content: overwritten
    b_dec.add_ref_feature_from_frame(ref_frame(H, W, seed=9), False)
    bits, ecp = a_enc.compress(chunk(H, W, 0), 21, False, pb, pr)
    a_dec.decompress(bits, 21, H, W, ecp, False)
    se, fe = a_enc.export_state()
    sdc, fd = a_dec.export_state()
    assert se.numel() == a_enc.state_bytes() > 0
    b_enc.import_state(se, fe)
    b_dec.import_state(sdc, fd)
    x = chunk(H, W, 8)
    bits_a, ecp_a = a_enc.compress(x, 42, False, pb, pr)
    bits_b, ecp_b = b_enc.compress(x, 42, False, pb, pr)
    assert ecp_a == ecp_b and np.array_equal(bits_a, bits_b)
    fa = [f.clone() for f in a_dec.decompress(bits_a, 42, H, W, ecp_a, False)]
    fb = b_dec.decompress(bits_b, 42, H, W, ecp_b, False)
    torch.cuda.synchronize()
    assert all(torch.equal(x1, x2) for x1, x2 in zip(fa, fb))
    # a codec that shares the parameters allocates no parameter copy of its own (HT-S: ~160 MB)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    c = DMCHTSProxy()
    c.share_params_from(a_enc)
    torch.cuda.synchronize()
    assert free0 - torch.cuda.mem_get_info()[0] < 32 * 2 ** 20
