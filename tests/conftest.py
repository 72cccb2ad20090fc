"""Shared fixtures.  GPU tests carry @pytest.mark.gpu; everything else runs on CPU."""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))

GOLDEN_DIR = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 (B200) GPU")


class Golden:
    def __init__(self):
        self.results = json.loads((GOLDEN_DIR / "golden.json").read_text())
        self.arrays = np.load(GOLDEN_DIR / "golden.npz")

    def mats(self, name):
        r = self.results[name]
        return tuple(self.arrays[f"{name}__{i}"] for i in range(r["nmats"]))

    def names(self, kind=None):
        return [k for k, v in self.results.items() if kind is None or v["kind"] == kind]


@pytest.fixture(scope="session")
def golden():
    return Golden()


@pytest.fixture(scope="session")
def orc():
    from oracle.refbind import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def ref():
    from oracle.refbind import Ref, ref_available
    return Ref() if ref_available() else None


@pytest.fixture(scope="session")
def native():
    from qubitserf_b200 import _native
    _native.lib()
    return _native
