"""The header-only C++ drop-in (include/mccfr_trainer.hpp): a caller written
in the reference's main.cpp style compiles unchanged against it, fails with an
exception instead of exit(1) when no device exists, and trains, exports and
round-trips a checkpoint on the GPU."""
from __future__ import annotations

import json
import shutil
import subprocess
from pathlib import Path

import pytest

from conftest import PKG_DIR, ROOT, gpu_available

SRC = Path(__file__).with_name("drop_in_main.cpp")


def build(tmp_path: Path) -> Path:
    exe = tmp_path / "drop_in_main"
    cmd = ["g++", "-O2", "-std=c++17", str(SRC), f"-I{ROOT / 'include'}", f"-L{PKG_DIR}", "-lmccfr",
           f"-Wl,-rpath,{PKG_DIR}", "-o", str(exe)]
    subprocess.run(cmd, check=True)
    return exe


def run(exe: Path, tmp_path: Path, iters: int) -> dict:
    out = subprocess.run([str(exe), str(tmp_path), str(iters)], check=True, capture_output=True, text=True,
                         timeout=600).stdout
    return json.loads(out.strip().splitlines()[-1])


@pytest.mark.skipif(shutil.which("g++") is None, reason="no C++ compiler")
@pytest.mark.skipif(gpu_available(), reason="checks the no-device path")
def test_compiles_and_reports_missing_device(tmp_path):
    r = run(build(tmp_path), tmp_path, 1)
    assert "exception" in r and "no CUDA device" in r["exception"]


@pytest.mark.gpu
def test_trains_exports_and_restores(tmp_path):
    r = run(build(tmp_path), tmp_path, 2)
    assert "exception" not in r, r
    assert r["saved"] and r["loaded"] and r["same"]
    assert r["strategies"] > 0 and r["active"] > 0
