"""Shared test setup: import paths, the gpu marker, golden fixtures, GPU handles with tables."""

from __future__ import annotations

import json
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT / "cuda-cube-solver_b200"))
sys.path.insert(0, str(ROOT / "oracle"))
GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")


def load_golden(name: str):
    return json.loads((GOLDEN / name).read_text())


@pytest.fixture(scope="session")
def host_golden():
    return load_golden("host_model.json")


@pytest.fixture(scope="session")
def depth_golden():
    return load_golden("depth_counts.json")


@pytest.fixture(scope="session")
def lengths_golden():
    return load_golden("optimal_lengths.json")


@pytest.fixture(scope="session")
def oracle():
    from oracle import Oracle

    return Oracle()


_HANDLES = {}


def resident_handle(kind: str, fmt: str = "block"):
    """A libccs handle with ``kind`` built on the GPU and kept resident (once per session)."""

    from cuda_cube_solver import native

    key = (kind, fmt)
    if key not in _HANDLES:
        h = native.Handle()
        counts, secs = h.build_table(kind, fmt, None, keep_resident=True)
        h.build_counts, h.build_seconds = counts, secs
        _HANDLES[key] = h
    return _HANDLES[key]


def pytest_sessionfinish(session, exitstatus):
    for h in _HANDLES.values():
        h.close()
    _HANDLES.clear()
