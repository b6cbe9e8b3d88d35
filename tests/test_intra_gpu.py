"""GPU intra (DMCI) codec through the drop-in DMCIProxy: exact encoder/decoder round trips,
QP dependence, determinism, corrupt-stream errors, and parity with the FP64 oracle
(oracle/intra_oracle.py) on the same seeded weights and frames.

Parity tolerances (north-star targets): |PSNR_gpu - PSNR_oracle| <= 0.05 dB,
|bytes_gpu - bytes_oracle| <= 1 %, at least 97 % of the quantised y latents equal."""
import os
import sys

import numpy as np
import pytest
import torch

from dcvc_b200 import synthetic
from dcvc_b200._native import DcvcError
from tests.intra_fixtures import intra_frame, intra_state_dict, make_intra_proxy

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(__file__)), "oracle"))
import hts_oracle  # noqa: E402
import intra_oracle  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def sd16():
    return intra_state_dict()


@pytest.mark.parametrize("H,W", [(256, 256), (200, 248), (64, 1088)])
def test_round_trip_exact(sd16, H, W):
    enc, dec = make_intra_proxy(sd16), make_intra_proxy(sd16)
    x, _ = intra_frame(H, W)
    pr, pb = synthetic.padding_for(H, W)
    bits, x_hat, ecp = enc.compress(x, 32, pb, pr)
    assert bits.dtype == np.uint8 and bits.size > 0
    assert x_hat.shape == (1, 3, H + pb, W + pr)
    x_dec = dec.decompress(bits, 32, H, W, ecp)
    torch.cuda.synchronize()
    assert torch.equal(x_hat, x_dec)
    assert torch.equal(enc.buffer("y_hat"), dec.buffer("y_hat"))
    assert torch.equal(enc.buffer("z_hat"), dec.buffer("z_hat"))
    assert float(x_hat.abs().max()) <= 0.5
    sym, kernels, dev_bytes = enc.stats()
    assert sym > 0 and kernels > 100 and dev_bytes > 0


def test_graph_replay_and_qp_dependence(sd16):
    enc, dec = make_intra_proxy(sd16), make_intra_proxy(sd16)
    x, _ = intra_frame(256, 256)
    sizes = {}
    for qp in (0, 63, 0, 63, 0):   # eager, captured, replayed
        bits, x_hat, ecp = enc.compress(x, qp, 0, 0)
        x_hat = x_hat.clone()
        x_dec = dec.decompress(bits, qp, 256, 256, ecp)
        assert torch.equal(x_hat, x_dec), qp
        sizes.setdefault(qp, set()).add(bits.tobytes())
    assert len(sizes[0]) == 1 and len(sizes[63]) == 1   # deterministic across replays
    assert sizes[0] != sizes[63]


def test_resolution_change(sd16):
    enc, dec = make_intra_proxy(sd16), make_intra_proxy(sd16)
    for H, W in ((128, 128), (192, 320), (128, 128)):
        x, _ = intra_frame(H, W)
        bits, x_hat, ecp = enc.compress(x, 10, 0, 0)
        assert torch.equal(x_hat.clone(), dec.decompress(bits, 10, H, W, ecp))


def test_corrupt_stream_raises(sd16):
    enc, dec = make_intra_proxy(sd16), make_intra_proxy(sd16)
    x, _ = intra_frame(128, 128)
    bits, _, ecp = enc.compress(x, 20, 0, 0)
    with pytest.raises(DcvcError):
        dec.decompress(bits[: max(1, bits.size // 4)], 20, 128, 128, ecp)
    # the handle stays usable
    x_dec = dec.decompress(bits, 20, 128, 128, ecp)
    assert x_dec.shape == (1, 3, 128, 128)


def test_bad_arguments(sd16):
    enc = make_intra_proxy(sd16)
    x, _ = intra_frame(120, 128)
    with pytest.raises(DcvcError):
        enc.compress(x, 32, 0, 0)   # 120 is not a multiple of 16 without padding
    with pytest.raises(DcvcError):
        enc.compress(x, 64, 8, 0)   # qp out of range


@pytest.mark.parametrize("H,W,qp", [(256, 256, 32), (200, 248, 0), (128, 192, 63)])
def test_gpu_matches_fp64_oracle(sd16, H, W, qp):
    sd_cpu = {k: v.cpu() for k, v in sd16.items()}
    o = intra_oracle.IntraOracle(sd_cpu, 0.15, torch.float64)
    enc = make_intra_proxy(sd16)
    x, (y, u, v) = intra_frame(H, W)
    pr, pb = synthetic.padding_for(H, W)
    bits, x_hat, ecp = enc.compress(x, qp, pb, pr)
    gq = enc.buffer("y_q").float().cpu()
    r = o.compress(x.cpu(), qp, pb, pr)
    oq = r["y_q"][0].permute(1, 2, 0).reshape(-1, 256).float()
    agree = float((gq == oq).float().mean())
    pg = hts_oracle.psnr_yuv420(x_hat.float(), y, u, v)[0]
    po = hts_oracle.psnr_yuv420(r["x_hat"], y, u, v)[0]
    assert abs(pg - po) <= 0.05, (pg, po)
    ob = r["bit_stream"].size
    assert abs(bits.size - ob) <= 0.01 * ob, (bits.size, ob)
    assert agree >= 0.97, agree
