"""Shared pytest configuration: the ``gpu`` marker, repository imports and golden fixtures."""
import hashlib
import json
import sys
from pathlib import Path

import numpy as np
import pytest

REPO = Path(__file__).resolve().parent.parent
GOLDEN = REPO / "tests" / "golden"
if str(REPO) not in sys.path:
    sys.path.insert(0, str(REPO))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


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


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


class Golden:
    """Reader of one tests/golden/<stem>.{npz,json} pair written by make_golden.py."""

    def __init__(self, stem):
        self.meta = json.loads((GOLDEN / f"{stem}.json").read_text())
        self.z = np.load(GOLDEN / f"{stem}.npz")

    def names(self, prefix=""):
        return sorted(k for k in self.meta if k.startswith(prefix))

    def mask(self, name):
        shape = tuple(self.meta[name]["shape"])
        bits = self.z[f"{name}__mask"]
        return np.unpackbits(bits, count=int(np.prod(shape))).astype(bool).reshape(shape)

    def matches(self, name, key, actual):
        """True when ``actual`` equals the reference capture bit for bit."""
        return sha(actual) == self.meta[name]["sha256"][key]

    def array(self, name, key):
        k = f"{name}__{key}"
        return self.z[k] if k in self.z.files else None


@pytest.fixture(scope="session")
def golden():
    return Golden
