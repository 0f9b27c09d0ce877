"""Shared fixtures: golden cases from the reference, the oracle, and GPU availability."""

from __future__ import annotations

import json
from pathlib import Path
import sys

import numpy as np
import pytest

REPO = Path(__file__).resolve().parents[1]
GOLDEN = REPO / "tests" / "golden"
for path in (REPO, REPO / "oracle", REPO / "tests"):
    if str(path) not in sys.path:
        sys.path.insert(0, str(path))

# Tolerance for real-valued inputs when heavy rows are tree-reduced (default mode): the
# result differs from the reference's left-to-right sums only by reassociation.
RTOL_F64, ATOL_F64 = 1e-12, 1e-12
RTOL_F32, ATOL_F32 = 1e-5, 1e-5


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libgrg_b200.so")


def golden_index() -> list[dict]:
    return json.loads((GOLDEN / "cases_index.json").read_text())


@pytest.fixture(scope="session")
def golden_data():
    with np.load(GOLDEN / "cases.npz") as data:
        yield {k: data[k] for k in data.files}


def golden_inputs(case: dict, data: dict):
    key = case["key"]
    x = data[key + "|x"]
    init = None
    if case["init"] == "xtx":
        init = "xtx"
    elif case["init"]:
        init = data[key + "|init"]
    miss = data[key + "|miss_in"].copy() if case["miss"] else None
    return x, init, miss


def artifact_path(name: str) -> Path:
    return GOLDEN / f"{name}.grg_spmv"
