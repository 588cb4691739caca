"""Shared test set-up: registers the package as `mccfr_b200`, builds the
libraries when their sources changed, and provides the rank table."""
from __future__ import annotations

import importlib.util
import os
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
PKG_DIR = ROOT / "parallel-mccfr-for-multiplayer-nlh_b200"
sys.path.insert(0, str(ROOT / "oracle"))


def load_package():
    if "mccfr_b200" in sys.modules:
        return sys.modules["mccfr_b200"]
    spec = importlib.util.spec_from_file_location("mccfr_b200", PKG_DIR / "__init__.py",
                                                  submodule_search_locations=[str(PKG_DIR)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["mccfr_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def _build():
    spec = importlib.util.spec_from_file_location("mccfr_b200_build", PKG_DIR / "build.py")
    b = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(b)
    b.build_all()


_build()
mccfr = load_package()


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def hand_table() -> np.ndarray:
    return mccfr.hand_table()


@pytest.fixture(scope="session")
def hand_table_file(hand_table, tmp_path_factory) -> Path:
    p = tmp_path_factory.mktemp("handranks") / "handranks.dat"
    hand_table.tofile(p)
    return p


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
