"""The drop-in modules under the reference's names: the reference's own entropy models, run with
dcvc_b200's MLCodec_extensions_cpp, build the same CDF tables and code the same bytes as with the
reference's compiled module.  Runs only where the reference checkout is named by the
DCVC_REFERENCE environment variable (this checks the boundary from the reference's side; it is
skipped elsewhere)."""
import os
import sys

import numpy as np
import pytest
import torch

REF = os.environ.get("DCVC_REFERENCE", "")
pytestmark = pytest.mark.skipif(not REF or not os.path.isdir(os.path.join(REF, "src")),
                                reason="reference sources not available")


def test_reference_entropy_models_on_dropin_coder():
    from dcvc_b200 import dropin
    dropin.install()
    sys.path.insert(0, REF)
    try:
        from src.models.video_model_ht import DMC
        from src.utils.common import ModelStructure
        torch.manual_seed(0)
        m = DMC(ModelStructure.HTS)
        m.update(0.15)
        g = np.load(os.path.join(os.path.dirname(__file__), "golden", "cdf_tables.npz"))
        qy, ly = m.gaussian_encoder.get_cdf_info()
        qz, lz = m.bit_estimator_z.get_cdf_info()
        assert (qy == g["qy"]).all() and (ly == g["ly"]).all()
        assert (qz == g["qz"]).all() and (lz == g["lz"]).all()
        # the reference's EntropyCoder wrapper drives the drop-in RansEncoder / RansDecoder
        enc = m.entropy_coder.encoder
        rng = np.random.default_rng(0)
        ysym = ((rng.integers(-3, 4, 5000) << 8) + rng.integers(0, 128, 5000)).astype(np.int16)
        enc.set_entropy_coder_parallel(3)
        enc.reset()
        enc.encode_y(ysym)
        enc.flush()
        data = enc.get_encoded_stream()
        dec = m.entropy_coder.decoder
        dec.set_entropy_coder_parallel(3)
        dec.set_stream(data)
        dec.decode_y((ysym & 0xff).astype(np.uint8))
        assert (dec.get_decoded_tensor() == (ysym >> 8)).all()
    finally:
        dropin.uninstall()
        sys.path.remove(REF)
        for k in [k for k in sys.modules if k == "src" or k.startswith("src.")]:
            del sys.modules[k]
