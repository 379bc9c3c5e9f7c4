import glob
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "t-flows_b200"))

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def golden_cases():
    out = []
    for p in sorted(glob.glob(os.path.join(GOLDEN, "*.npz"))):
        d = dict(np.load(p, allow_pickle=False))
        d = {k: (v.item() if v.shape == () else v) for k, v in d.items()}
        d["name"] = os.path.basename(p)[:-4]
        d["norm"] = None if np.isnan(d["norm"]) else float(d["norm"])
        out.append(d)
    return out


@pytest.fixture(scope="session")
def gpu_ctx():
    from tflows_b200 import native
    ctx = native.Context(0)
    yield ctx
    ctx.close()
