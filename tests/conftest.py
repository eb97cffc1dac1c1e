"""Shared test set-up: the `gpu` marker, fixture loading, repository paths."""
from __future__ import annotations

import os
import sys

import numpy as np
import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 GPU (run with -m gpu on a B200)")


_cache: dict[str, dict] = {}


def golden(name: str) -> dict:
    """Arrays of tests/golden/<name>.npz (written by tests/golden/make_golden.py)."""
    if name not in _cache:
        with np.load(os.path.join(GOLDEN, f"{name}.npz")) as z:
            _cache[name] = {k: z[k] for k in z.files}
    return _cache[name]


def cases(name: str, prefix: str) -> list[str]:
    """Keys '<prefix>/.../end' of a golden file, without the '/end'."""
    return sorted(k[: -len("/end")] for k in golden(name) if k.startswith(prefix) and k.endswith("/end"))


@pytest.fixture(scope="session")
def gpu_lib():
    from randomtilings_b200 import _capi

    return _capi.load()
