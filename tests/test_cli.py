"""The command-line front end (mccfr_cli): the reference's flags
(poker_cuda/src/main.cpp:29-69), a clean report without a GPU, and on the GPU a
training run that writes the reference's v2 strategy dump and checkpoint."""
from __future__ import annotations

import re
import subprocess

import numpy as np
import pytest

from conftest import PKG_DIR, gpu_available

CLI = PKG_DIR / "mccfr_cli"


def run(*args: str, timeout: int = 600) -> subprocess.CompletedProcess:
    return subprocess.run([str(CLI), *args], capture_output=True, text=True, timeout=timeout)


def test_usage_lists_the_reference_flags():
    r = run("--help")
    assert r.returncode == 0
    for flag in ("--mode", "--players", "--iters", "--batch", "--stack", "--sb", "--bb", "--save", "--load",
                 "--handranks", "--no-cfrplus", "--cfrplus", "--no-lcfr", "--lcfr"):
        assert flag in r.stdout, flag
    assert "train|benchmark|info" in r.stdout


@pytest.mark.skipif(gpu_available(), reason="checks the no-device path")
def test_info_without_gpu():
    r = run("--mode", "info")
    assert r.returncode == 0 and "GPUs found: 0" in r.stdout


@pytest.mark.gpu
def test_train_writes_reference_dump_and_checkpoint(tmp_path):
    save = tmp_path / "strategy.bin"
    r = run("--mode", "train", "--iters", "2", "--batch", "2048", "--save", str(save),
            "--handranks", str(tmp_path / "absent.dat"))  # a missing table is generated
    assert r.returncode == 0, r.stdout + r.stderr
    active = int(re.search(r"Info sets active: (\d+)", r.stdout).group(1))
    assert active > 0
    raw = save.read_bytes()
    magic = np.frombuffer(raw[:8], np.uint64)[0]
    ts, na, n = np.frombuffer(raw[8:20], np.uint32)
    assert (magic, ts, na) == (0x53545241540100, 1 << 26, 8)
    assert n > 0 and len(raw) == 20 + int(n) * 36
    probs = np.frombuffer(raw[20:], dtype=np.dtype([("k", np.uint32), ("p", np.float32, 8)]))["p"]
    assert np.allclose(probs.sum(1), 1.0, atol=1e-5)
    ck = tmp_path / "strategy.bin.ckpt"
    assert ck.stat().st_size == 16 + 2 * 8 * (1 << 26) * 4  # the reference's checkpoint layout
