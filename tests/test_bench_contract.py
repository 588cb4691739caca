"""bench.py's output contract, on the CPU: the reference arm prints one JSON line
with the keys the driver reads, other ranks of a multi-rank launch print nothing
and exit 0, and the helper figures are computed as documented."""
from __future__ import annotations

import json
import os
import subprocess
import sys
from types import SimpleNamespace

import pytest

from conftest import ROOT

KEYS = {"impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
        "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"}


def bench(*args: str, env: dict | None = None) -> subprocess.CompletedProcess:
    e = dict(os.environ)
    e.update(env or {})
    return subprocess.run([sys.executable, str(ROOT / "bench.py"), *args], capture_output=True, text=True,
                          timeout=900, env=e, cwd=str(ROOT))


def test_reference_arm_line():
    r = bench("--impl", "reference", "--workload", "hu-20bb", "--steps", "1", "--warmup", "1")
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [x for x in r.stdout.splitlines() if x.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert KEYS <= set(d)
    assert d["impl"] == "reference" and d["unit"] == "traversals/s" and d["higher_is_better"] is True
    assert d["value"] > 0 and d["e2e"]["value"] == d["value"] and d["cpu_baseline"]["value"] == d["value"]
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] >= 1
    assert d["config"]["workload"] == "hu-20bb" and d["steps"] == 1 and d["warmup"] == 1
    assert "visits per traversal" in d["cpu_baseline"]["sample"]


def test_reference_arm_other_ranks_are_silent():
    r = bench("--impl", "reference", "--steps", "1", "--warmup", "1", env={"RANK": "1", "WORLD_SIZE": "2"})
    assert r.returncode == 0 and r.stdout.strip() == ""


def test_apply_roofline_and_sample_text():
    sys.path.insert(0, str(ROOT))
    import bench as b

    s0 = SimpleNamespace(apply_ms=1.0, touched_last=0)
    s1 = SimpleNamespace(apply_ms=11.0, touched_last=1_000_000)
    a = b.apply_roofline(s0, s1, 2, 6000.0)
    assert a["kernel_ms_per_launch"] == 5.0
    assert a["achieved"] == pytest.approx(1_000_000 * 516 / 0.005 / 1e9)
    assert a["frac"] == pytest.approx(a["achieved"] / 6000.0)
    info = {"seconds": 2.0, "cores": 8, "visits_per_traversal": 1040.0, "visits_per_s": 8.5e6,
            "raw_traversals_per_s": 8000.0}
    assert "55.32" in b.cpu_sample_text(16384, info, 55.32)
    assert "raw traversals/s" in b.cpu_sample_text(16384, info, None)
    assert b.work_per_traversal("6max-100bb") == pytest.approx(55.32)
    assert b.work_per_traversal("no-such-workload") is None
