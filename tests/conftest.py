"""Shared test helpers.

Markers: ``gpu`` -- needs a CUDA device (run with ``-m gpu`` on a B200).
Everything else runs on CPU.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

REPO = Path(__file__).resolve().parent.parent
GOLDEN = REPO / "tests" / "golden"
if str(REPO) not in sys.path:
    sys.path.insert(0, str(REPO))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: test needs a CUDA GPU (B200)")


def load_golden(name: str):
    """(SpinSystem built from the reference's own arrays, raw fixture dict)."""
    from oracle import oracle as O
    d = dict(np.load(GOLDEN / f"{name}.npz"))
    return O.system_from_dump(d), d


def ref_spins(d: dict, step: int) -> np.ndarray:
    return np.stack([d[f"sx_{step}"], d[f"sy_{step}"], d[f"sz_{step}"]])


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def vgpu_lib():
    """libvgpu.so, built in-tree if missing (a GPU run must use the CUDA path)."""
    from vampire_b200 import build, vgpu
    build.build()
    return vgpu.lib()
