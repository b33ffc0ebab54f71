"""Shared pytest configuration.

Markers: ``gpu`` tests need a CUDA device (B200) and call the CUDA path
through libjqc.so; everything else runs on CPU.  ``golden`` loads the
fixtures in tests/golden (made by running the reference's own code, see
tests/golden/gen_golden.py)."""

from __future__ import annotations

import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device; runs the sm_100a kernels")


class Golden:
    def __init__(self, tag):
        self.rec = json.load(open(os.path.join(GOLDEN, tag + ".json")))
        self.arr = np.load(os.path.join(GOLDEN, tag + ".npz"), allow_pickle=True)

    def molecule(self):
        from jax_examples_b200.core import make_molecule

        r = self.rec
        return make_molecule(tuple(r["elements"]), np.array(r["coords"]), np.array(r["Z"]),
                             charge=r["charge"], spin=r["spin"])

    def basis(self):
        from jax_examples_b200.basis import build_basis_set

        return build_basis_set(self.molecule(), self.rec["basis"], spherical=bool(self.rec.get("spherical", False)))


@pytest.fixture(scope="session")
def golden():
    cache = {}

    def get(tag):
        if tag not in cache:
            cache[tag] = Golden(tag)
        return cache[tag]

    return get


@pytest.fixture(scope="session")
def libjqc():
    """libjqc.so, built in-tree if it is missing."""
    from jax_examples_b200 import _abi, _build

    if not os.path.exists(_abi.LIB_PATH):
        _build.build()
    return _abi.load()
