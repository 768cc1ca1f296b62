import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

ULP = np.finfo(np.float64).eps


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


def pytest_collection_modifyitems(config, items):
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:  # pragma: no cover
        has_gpu = False
    if has_gpu:
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


@pytest.fixture(scope="session")
def golden():
    path = os.path.join(ROOT, "tests", "golden", "green_apply_golden.npz")
    with np.load(path) as f:
        data = {k: f[k] for k in f.files}
    return data


def golden_cases(data):
    from tests.golden.make_golden import parse, unit_block
    out = []
    for key in data["names"]:
        key = str(key)
        variant, shape, _, block, offs = parse(key + ".npz")
        comp = int(data[key + "/comp"])
        out.append((key, variant, shape, comp, block, offs))
    return out


def reference_checker():
    """The reference's Cython modules built against the FFT shim, if built
    (oracle/_ref); None otherwise."""
    from oracle import reference
    return reference.load()
