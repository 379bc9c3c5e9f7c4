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


def _load(p):
    d = dict(np.load(p, allow_pickle=False))
    d = {k: (v.item() if v.shape == () else v) for k, v in d.items()}
    d["name"] = os.path.basename(p)[:-4]
    d["norm"] = None if np.isnan(d["norm"]) else float(d["norm"])
    return d


def generated_cases():
    """Fixtures stored as a generator call (inputs rebuilt here, checked by
    their SHA-256) plus the reference source's outputs."""
    return [_load(p) for p in sorted(glob.glob(os.path.join(GOLDEN, "gen_*.npz")))]


def build_generated(case):
    """System of a generated fixture, rebuilt by the generator it names;
    fails if the generator's inputs drifted from the recorded SHA-256."""
    from golden.make_golden import input_sha
    from tflows_b200 import systems
    gen = case["generator"]
    if not gen.startswith("ldc_pressure_30("):
        raise ValueError(gen)
    singular = "pin" if "singular='pin'" in gen else "set_singular"
    s = systems.ldc_pressure_30(seed=1, singular=singular)
    sha = input_sha(s.csr.row, s.csr.col, s.csr.dia, s.val, s.b, s.x0)
    assert sha == case["input_sha256"], f"{case['name']}: the generator's inputs changed"
    return s


def golden_cases():
    out = []
    for p in sorted(glob.glob(os.path.join(GOLDEN, "*.npz"))):
        if os.path.basename(p).startswith("gen_"):
            continue
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
