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


def config_json(*args: str) -> tuple[int, dict, str]:
    import json

    r = run("--mode", "config", *args)
    return r.returncode, (json.loads(r.stdout.strip().splitlines()[-1]) if r.stdout.strip() else {}), r.stderr


def test_config_mode_defaults_to_the_reference_game():
    rc, c, _ = config_json()
    assert rc == 0 and c["valid"]
    assert (c["players"], c["stack"], c["sb"], c["bb"], c["seed"]) == (2, 1000, 10, 20, 42)
    assert c["actions"] == ["fold", "check", "call", "min_raise", "1/2", "2/3", "1/1", "all_in"]
    assert c["keys"] == "fnv26" and c["table_log2"] == 26 and c["max_depth"] == 20


def test_config_file_then_flags(tmp_path):
    f = tmp_path / "game.cfg"
    f.write_text("""# heads-up 50BB, three sizes
preset = hu20
players = 2
stack = 5000      # chips: 1 BB = 100
actions = fold, check_call, 1/3, 3/4, 3/2, all_in
raise_cap = 3
postflop_buckets = 30, 40, 50
cfr_plus = false
seed = 7
""")
    rc, c, _ = config_json("--config", str(f), "--seed", "9", "--raise-cap", "1")
    assert rc == 0 and c["valid"]
    assert c["stack"] == 5000 and c["cfr_plus"] == 0 and c["lcfr"] == 1
    assert c["actions"] == ["fold", "check_call", "1/3", "3/4", "3/2", "all_in"]
    assert c["postflop_buckets"] == [30, 40, 50] and c["keys"] == "id64"
    assert c["seed"] == 9 and c["raise_cap"] == 1  # flags override the file


def test_config_errors(tmp_path):
    bad = tmp_path / "bad.cfg"
    bad.write_text("players = 9\n")
    rc, c, _ = config_json("--config", str(bad))
    assert rc == 1 and not c["valid"] and "players" in c["why"]
    for text, msg in (("colour = red\n", "unknown config key"), ("players\n", "expected key = value"),
                      ("actions = fold, shove\n", "bad value")):
        bad.write_text(text)
        rc, _, err = config_json("--config", str(bad))
        assert rc == 1 and msg in err, (text, err)
