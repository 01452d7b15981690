"""pytest configuration: the `gpu` marker and import helpers for the package and the oracle.

Tests marked gpu run on a B200 (the library's kernels); the rest run on CPU.  The oracle
under oracle/ is test infrastructure and is only used here as the checker.
"""
from __future__ import annotations

import importlib.util
import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_DIR = os.path.join(ROOT, "two-phase-3equation-2d-pal-column_b200")
GOLDEN = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def import_package():
    """the package directory name has hyphens, so it is imported from its path"""
    if "wenofv_b200" in sys.modules:
        return sys.modules["wenofv_b200"]
    spec = importlib.util.spec_from_file_location("wenofv_b200", os.path.join(PKG_DIR, "__init__.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules["wenofv_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def golden_cases():
    with open(os.path.join(GOLDEN, "index.json")) as f:
        return json.load(f)


def load_golden(name):
    with np.load(os.path.join(GOLDEN, name + ".npz")) as z:
        return {k: z[k] for k in z.files}


@pytest.fixture(scope="session")
def wb():
    return import_package()


@pytest.fixture(scope="session")
def oracle_lib():
    from oracle import Oracle
    return Oracle()
