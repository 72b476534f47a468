"""Shared fixtures.  Tests marked `gpu` need a CUDA device; everything else runs on CPU."""
from __future__ import annotations

import json
import pathlib
import sys

import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden"
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))

import __graft_entry__  # noqa: E402


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device")


@pytest.fixture(scope="session")
def pg():
    return __graft_entry__.load_package()


@pytest.fixture(scope="session")
def oracle():
    import oracle as O
    O.build()
    return O


@pytest.fixture(scope="session")
def ctx(pg):
    c = pg.Context(0)
    yield c
    c.close()


def golden(name: str) -> dict:
    return json.loads((GOLDEN / name).read_text())


@pytest.fixture(scope="session")
def prp_vectors():
    return golden("prp_vectors.json")
