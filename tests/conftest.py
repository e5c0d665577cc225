"""Test configuration: the `gpu` marker, and an in-tree build of the library
(and of the C oracle) before any test loads them."""
from __future__ import annotations

import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def pytest_sessionstart(session):
    from master_b200 import build
    build.build()
    subprocess.run(["make", "-s", "-C", str(ROOT / "oracle"), "oracle"], check=True)


def has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
