import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from ginkgo_b200.stencils import std_uniform  # noqa: E402,F401


def pytest_configure(config):
    config.addinivalue_line(
        "markers", "gpu: needs a CUDA device (B200); runs the CUDA library")


@pytest.fixture(scope="session")
def known():
    with open(os.path.join(ROOT, "tests", "golden", "known_answers.json")) as f:
        return json.load(f)


def to_array(a, dtype=np.float64):
    """JSON lists with the string "nan" -> numpy array."""
    return np.array([[np.nan if v == "nan" else v for v in row]
                     if isinstance(row, list) else
                     (np.nan if row == "nan" else row) for row in a],
                    dtype=dtype)


def dense_to_csr(d):
    d = np.asarray(d, dtype=np.float64)
    rp = [0]
    ci, v = [], []
    for row in d:
        nz = np.nonzero(row)[0]
        ci.extend(nz.tolist())
        v.extend(row[nz].tolist())
        rp.append(len(ci))
    return (np.array(rp, np.int32), np.array(ci, np.int32),
            np.array(v, np.float64))
