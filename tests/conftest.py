"""Shared pytest configuration: the `gpu` marker and common fixtures."""
import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def ref_table():
    with open(os.path.join(GOLDEN, "reference_primes.json")) as f:
        return json.load(f)


@pytest.fixture
def rng():
    return np.random.default_rng(1234)
