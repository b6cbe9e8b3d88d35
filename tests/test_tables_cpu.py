"""Seeded weights and CDF tables against the reference's (golden fixtures from make_golden.py)."""
import json
import os

import numpy as np
import pytest

from dcvc_b200.entropy_tables import bit_estimator_tables, gaussian_tables
from dcvc_b200.model_spec import hts_state_dict

GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module")
def sd0():
    return hts_state_dict(0)


def test_seed0_weights_equal_reference(sd0):
    fp = json.load(open(os.path.join(GOLD, "weights_seed0.json")))
    assert list(sd0.keys()) == list(fp.keys())
    for k, v in sd0.items():
        t = v.double().reshape(-1)
        f = fp[k]
        assert list(v.shape) == f["shape"], k
        assert [float(x) for x in t[:4]] == f["head"], k
        assert abs(float(t.sum()) - f["sum"]) <= 1e-9 * max(1.0, abs(f["sum"])), k
        assert abs(float((t * t).sum()) - f["sumsq"]) <= 1e-9 * max(1.0, f["sumsq"]), k
    assert sum(v.numel() for v in sd0.values()) == 81157632


def test_gaussian_tables_equal_reference():
    g = np.load(os.path.join(GOLD, "cdf_tables.npz"))
    qy, ly = gaussian_tables()
    assert (qy == g["qy"]).all() and (ly == g["ly"]).all()


def test_bit_estimator_tables_equal_reference(sd0):
    g = np.load(os.path.join(GOLD, "cdf_tables.npz"))
    qz, lz = bit_estimator_tables(sd0["bit_estimator_z.h"], sd0["bit_estimator_z.b"],
                                  sd0["bit_estimator_z.a"])
    assert (qz == g["qz"]).all() and (lz == g["lz"]).all()
