"""GPU rANS coder: payload bytes identical with the reference coder's golden bytes and with the
host coder over many symbol sets, ec_parallel 1..8, bypass escapes and batches of payloads;
decoding back to the symbols; truncated and corrupt payloads report an error status."""
import numpy as np
import pytest
import torch

from dcvc_b200 import MLCodec_extensions_cpp as M
from dcvc_b200.entropy_tables import gaussian_tables
from dcvc_b200.rans_gpu import GpuRansCoder
from tests.test_rans_cpu import gold  # noqa: F401  (fixture)

pytestmark = pytest.mark.gpu


def _cpu_payload(qy, ly, qz, lz, y, z, qp, ecp):
    enc = M.RansEncoder()
    enc.set_cdf(qz, lz, 0)
    enc.set_cdf(qy, ly, 1)
    enc.set_entropy_coder_parallel(ecp)
    enc.reset()
    enc.encode_y(y)
    enc.encode_z(z, qp * 128, 128)
    enc.flush()
    return enc.get_encoded_stream()


def test_gpu_matches_reference_golden_bytes(gold):  # noqa: F811
    qy, ly, qz, lz, cases = gold
    g = GpuRansCoder(qz, lz, qy, ly)
    jobs = [{"y": torch.from_numpy(y.astype(np.int16)).cuda(), "z": torch.from_numpy(z.astype(np.int8)).cuda(),
             "z_offset": qp * 128, "z_ch": 128, "ecp": ecp} for ny, nz, ecp, qp, y, z, ref in cases]
    outs, st = g.encode(jobs)
    assert st == [0] * len(cases)
    for (ny, nz, ecp, qp, y, z, ref), o in zip(cases, outs):
        assert o.cpu().numpy().tobytes() == ref.tobytes(), (ny, nz, ecp)
    dec, st = g.decode([{"data": torch.from_numpy(ref).cuda(), "ecp": ecp, "n_z": nz,
                         "z_offset": qp * 128, "z_ch": 128,
                         "y_idx": torch.from_numpy((y & 0xff).astype(np.uint8)).cuda()}
                        for ny, nz, ecp, qp, y, z, ref in cases])
    assert st == [0] * len(cases)
    for (ny, nz, ecp, qp, y, z, ref), (zo, yo) in zip(cases, dec):
        assert np.array_equal(zo.cpu().numpy(), z.astype(np.int8))
        assert np.array_equal(yo.cpu().numpy(), (y >> 8).astype(np.int8))


def _random_job(rng, ny, nz, scale):
    q = np.clip(np.round(rng.laplace(0, scale, ny)), -128, 127).astype(np.int64)
    idx = rng.integers(0, 128, ny)
    y = ((q << 8) + idx).astype(np.int16)
    z = np.clip(np.round(rng.laplace(0, scale, nz)), -64, 63).astype(np.int8)
    return y, z


@pytest.mark.parametrize("seed", [0, 1])
def test_gpu_matches_host_coder_batched(gold, seed):  # noqa: F811
    _, _, qz, lz, _ = gold
    qy, ly = gaussian_tables()
    rng = np.random.default_rng(seed)
    g = GpuRansCoder(qz, lz, qy, ly)
    specs = []
    for k in range(24):
        ny = int(rng.integers(0, 300000)) if k % 5 else int(rng.integers(0, 50))
        nz = int(rng.integers(0, 20000))
        ecp = 1 + k % 8
        qp = int(rng.integers(0, 64))
        y, z = _random_job(rng, ny, nz, [0.5, 3.0, 30.0][k % 3])
        specs.append((y, z, qp, ecp))
    outs, st = g.encode([{"y": torch.from_numpy(y).cuda(), "z": torch.from_numpy(z).cuda(),
                          "z_offset": qp * 128, "z_ch": 128, "ecp": ecp} for y, z, qp, ecp in specs])
    assert st == [0] * len(specs)
    for (y, z, qp, ecp), o in zip(specs, outs):
        ref = _cpu_payload(qy, ly, qz, lz, y, z, qp, ecp)
        assert o.cpu().numpy().tobytes() == ref.tobytes(), (y.size, z.size, ecp)
    dec, st = g.decode([{"data": o, "ecp": ecp, "n_z": z.size, "z_offset": qp * 128, "z_ch": 128,
                         "y_idx": torch.from_numpy((y & 0xff).astype(np.uint8)).cuda()}
                        for (y, z, qp, ecp), o in zip(specs, outs)])
    assert st == [0] * len(specs)
    for (y, z, qp, ecp), (zo, yo) in zip(specs, dec):
        assert np.array_equal(zo.cpu().numpy(), z)
        assert np.array_equal(yo.cpu().numpy(), (y >> 8).astype(np.int8))


def test_corrupt_payloads_report_status(gold):  # noqa: F811
    _, _, qz, lz, _ = gold
    qy, ly = gaussian_tables()
    g = GpuRansCoder(qz, lz, qy, ly)
    rng = np.random.default_rng(5)
    y, z = _random_job(rng, 200000, 5000, 3.0)
    outs, st = g.encode([{"y": torch.from_numpy(y).cuda(), "z": torch.from_numpy(z).cuda(),
                          "z_offset": 0, "z_ch": 128, "ecp": 6}])
    assert st == [0]
    p = outs[0]
    idx = torch.from_numpy((y & 0xff).astype(np.uint8)).cuda()
    bad_header = p.clone()
    bad_header[0:4] = torch.tensor([255, 255, 255, 127], dtype=torch.uint8)
    _, st = g.decode([{"data": p[: p.numel() // 3], "ecp": 6, "n_z": z.size, "z_offset": 0,
                       "z_ch": 128, "y_idx": idx},
                      {"data": bad_header, "ecp": 6, "n_z": z.size, "z_offset": 0, "z_ch": 128,
                       "y_idx": idx}])
    assert st[0] in (3, 4) and st[1] == 3
    # a y symbol naming a table past the Gaussian set
    y_bad = y.copy()
    y_bad[7] = (y_bad[7] & ~0xff) | 200
    _, st = g.encode([{"y": torch.from_numpy(y_bad).cuda(), "z": torch.from_numpy(z).cuda(),
                       "z_offset": 0, "z_ch": 128, "ecp": 2}])
    assert st == [1]
