"""Shared fixtures: golden vectors, GPU marker, device helpers."""

from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = Path(__file__).resolve().parent / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def _load_cases():
    z = np.load(GOLDEN / "cases.npz")
    meta = json.loads(bytes(z["meta"]).decode())
    cases = []
    for i, m in enumerate(meta):
        cases.append(dict(m, idx=i, a=z[f"a{i}"], l=z[f"l{i}"], info=z[f"info{i}"]))
    return cases, z


_CASES, _Z = _load_cases()


@pytest.fixture(scope="session")
def golden_cases():
    return _CASES


@pytest.fixture(scope="session")
def golden_nonspd():
    return _Z["nonspd_a"], _Z["nonspd_info"]


@pytest.fixture(scope="session")
def golden_backward():
    z = np.load(GOLDEN / "backward.npz")
    out = []
    i = 0
    while f"a{i}" in z:
        out.append({k: z[f"{k}{i}"] for k in ("a", "l", "lbar", "abar")})
        i += 1
    return out


def case_id(c):
    return f"{c['case']}-b{c['batch']}-n{c['n']}"


GOLDEN_CASES = _CASES
