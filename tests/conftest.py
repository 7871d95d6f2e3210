"""Shared test set-up: import paths, the gpu marker, golden fixtures."""

from __future__ import annotations

import json
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
for p in (ROOT, ROOT / "sumcheck-triton_b200"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))

GOLDEN = Path(__file__).resolve().parent / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built library")


def load_jsonl(name: str) -> list[dict]:
    with open(GOLDEN / name) as f:
        return [json.loads(line) for line in f if line.strip()]


@pytest.fixture(scope="session")
def registry_records():
    return load_jsonl("registry_checksums.jsonl")


@pytest.fixture(scope="session")
def reference_outputs():
    return load_jsonl("reference_outputs.jsonl")


@pytest.fixture(scope="session")
def guard_cases():
    return load_jsonl("guard_cases.jsonl")
