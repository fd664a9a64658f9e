"""Test configuration: the `gpu` marker and shared fixtures."""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = Path(__file__).resolve().parent / "golden"
sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the CUDA path through the C ABI")


def golden(name: str):
    p = GOLDEN / name
    if p.suffix == ".json":
        return json.loads(p.read_text())
    return dict(np.load(p, allow_pickle=False))


def rows_from(nn, flat):
    out, k = [], 0
    for n in nn:
        out.append(np.asarray(flat[k:k + n], np.int64))
        k += n
    return out


def ewald_golden(name="ewald_xi0.5_err1e-3.npz"):
    g = golden(name)
    return g["table"], float(g["self_x"]), float(g["self_y"]), float(g["cut"]), int(g["n"])


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")
