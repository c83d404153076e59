import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
GOLDEN = os.path.join(ROOT, "tests", "golden")
# The reference sources, for CPU tests that read its files (absent on GPU hosts).
REFERENCE_DIR = os.environ.get("ASZ_REFERENCE_DIR", "/root/reference")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (run on a B200)")


def golden_cases():
    with open(os.path.join(GOLDEN, "manifest.json")) as f:
        return json.load(f)["cases"]


def load_golden(case):
    shape = tuple(case["shape"])
    data = np.fromfile(os.path.join(GOLDEN, case["name"] + ".f32"), np.float32).reshape(shape)
    with open(os.path.join(GOLDEN, case["name"] + ".asz"), "rb") as f:
        blob = f.read()
    out = np.fromfile(os.path.join(GOLDEN, case["name"] + ".out.f32"), np.float32).reshape(shape)
    return data, blob, out


@pytest.fixture(scope="session")
def gpu_ctx():
    import asz_b200.api as api
    ctx = api.Context(0)
    yield ctx
    ctx.close()
