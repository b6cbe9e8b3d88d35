"""Generates the golden fixtures under tests/golden/ from the reference itself.

Run here, where the reference sources exist (the reference checkout given by --ref or the DCVC_REFERENCE environment variable) and oracle/_ref has been
built by `make -C oracle`:

    python tests/golden/make_golden.py [--ref <reference checkout>]

Outputs (all small, committed):
  rans_golden.npz     symbols and the reference coder's bytes for ec_parallel 1..8 and edge cases
  pmf_golden.npz      pmfs and the reference pmf_to_quantized_cdf outputs
  cdf_tables.npz      the reference model's CDF tables after update(0.15) (HT-S, seed 0)
  weights_seed0.json  fingerprints of the reference HT-S state dict for torch.manual_seed(0)
  modules_golden.npz  reference nn.Module outputs for small inputs (pins the network oracle)
"""
import argparse
import ctypes
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def _ref_rans():
    return ctypes.PyDLL(os.path.join(ROOT, "oracle", "_ref", "librans_ref.so"))


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def make_cdf_tables(model):
    qy, ly = model.gaussian_encoder.get_cdf_info()
    qz, lz = model.bit_estimator_z.get_cdf_info()
    return (np.ascontiguousarray(qy, np.int32), np.ascontiguousarray(ly, np.int32),
            np.ascontiguousarray(qz, np.int32), np.ascontiguousarray(lz, np.int32))


def make_rans(qy, ly, qz, lz):
    ref = _ref_rans()
    rng = np.random.default_rng(1234)
    cases = [(20000, 2040, e, 7) for e in range(1, 9)]
    cases += [(0, 510, 1, 0), (0, 510, 4, 63), (5, 510, 8, 21), (1000, 0, 3, 42),
              (7, 3, 8, 1), (65536, 510, 2, 32)]
    out = {"qy": qy, "ly": ly}
    # keep the z tables of the QPs used by the cases only (the full table set is large)
    qps = sorted({c[3] for c in cases})
    out["qz_qps"] = np.array(qps, np.int32)
    out["qz"] = np.concatenate([qz[q * 128:(q + 1) * 128] for q in qps])
    out["lz"] = np.concatenate([lz[q * 128:(q + 1) * 128] for q in qps])
    for i, (ny, nz, ecp, qp) in enumerate(cases):
        idx = rng.integers(0, 128, ny)
        val = np.clip(np.round(rng.standard_normal(ny) * (idx / 127 * 8 + 0.3)), -128, 127)
        big = rng.random(ny) < 0.003
        val[big] = rng.integers(-128, 128, int(big.sum()))
        ysym = ((val.astype(np.int64) << 8) + idx).astype(np.int16)
        z = np.clip(np.round(rng.standard_normal(nz) * 6), -64, 63).astype(np.int8)
        z[:min(nz, 4)] = np.array([-64, 63, 0, -1], np.int8)[:min(nz, 4)]
        cap = (ny + nz) * 4 + 1024
        buf = np.zeros(cap, np.uint8)
        n = ref.ref_encode(_p(qz), _p(lz), qz.shape[0], qz.shape[1], _p(qy), _p(ly), qy.shape[0],
                           qy.shape[1], _p(ysym), ny, _p(z), nz, qp * 128, 128, ecp, _p(buf), cap)
        assert n > 0
        out[f"c{i}_meta"] = np.array([ny, nz, ecp, qp], np.int32)
        out[f"c{i}_y"] = ysym
        out[f"c{i}_z"] = z
        out[f"c{i}_bytes"] = buf[:n].copy()
    out["ncases"] = np.array(len(cases), np.int32)
    np.savez_compressed(os.path.join(HERE, "rans_golden.npz"), **out)


def make_pmf():
    ref = _ref_rans()
    rng = np.random.default_rng(99)
    pmfs = []
    for n in [3, 5, 7, 17, 18, 19]:
        p = rng.random(n).astype(np.float32)
        pmfs.append(p / p.sum())
    # tiny probabilities exercise the frequency-stealing branch
    p = np.full(18, 1e-7, np.float32)
    p[3] = 1.0 - 17e-7
    pmfs.append(p)
    p = np.array([0.5, 0.5 - 3e-6, 1e-6, 1e-6, 1e-6], np.float32)
    pmfs.append(p)
    out = {"n": np.array(len(pmfs), np.int32)}
    for i, p in enumerate(pmfs):
        cdf = np.zeros(p.size + 1, np.uint32)
        m = ref.ref_pmf_to_quantized_cdf(_p(p), p.size, _p(cdf))
        assert m == p.size + 1
        out[f"p{i}"] = p
        out[f"c{i}"] = cdf
    np.savez_compressed(os.path.join(HERE, "pmf_golden.npz"), **out)


def fingerprint(sd):
    fp = {}
    for k, v in sd.items():
        t = v.detach().double().reshape(-1)
        fp[k] = {"shape": list(v.shape), "sum": float(t.sum()), "sumsq": float((t * t).sum()),
                 "head": [float(x) for x in t[:4]]}
    return fp


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("DCVC_REFERENCE"),
                    help="reference checkout (default: $DCVC_REFERENCE)")
    args = ap.parse_args()
    if not args.ref:
        ap.error("give --ref or set DCVC_REFERENCE to the reference checkout")
    sys.path.insert(0, args.ref)
    sys.path.insert(0, os.path.join(ROOT, "oracle", "_ref"))
    import torch
    from src.models.video_model_ht import DMC
    from src.utils.common import ModelStructure

    torch.manual_seed(0)
    model = DMC(ModelStructure.HTS)
    sd = {k: v.clone() for k, v in model.state_dict().items()}
    with open(os.path.join(HERE, "weights_seed0.json"), "w") as f:
        json.dump(fingerprint(sd), f)
    model.update(0.15)
    qy, ly, qz, lz = make_cdf_tables(model)
    np.savez_compressed(os.path.join(HERE, "cdf_tables.npz"), qy=qy, ly=ly, qz=qz, lz=lz)
    make_rans(qy, ly, qz, lz)
    make_pmf()
    from make_modules_golden import make_modules
    make_modules(model)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    sys.path.insert(0, HERE)
    main()
