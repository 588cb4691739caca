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
    assert d["cpu_baseline"]["V_per_traversal"] > 1.0 and "timed iterations" in d["cpu_baseline"]["sample"]
    # the arm runs the oracle only: the product library is never loaded
    libs = d["libraries_loaded"]
    assert any(x.endswith("liboracle.so") for x in libs)
    assert not any(x.endswith("libmccfr.so") for x in libs)


def test_reference_arm_other_ranks_are_silent():
    r = bench("--impl", "reference", "--steps", "1", "--warmup", "1", env={"RANK": "1", "WORLD_SIZE": "2"})
    assert r.returncode == 0 and r.stdout.strip() == ""


def test_apply_roofline():
    sys.path.insert(0, str(ROOT))
    import bench as b

    s0 = SimpleNamespace(apply_ms=1.0, touched_last=0, wide_rows_last=0)
    s1 = SimpleNamespace(apply_ms=11.0, touched_last=1_000_000, wide_rows_last=250_000)
    a = b.apply_roofline(s0, s1, 2, 6000.0)
    assert a["kernel_ms_per_launch"] == 5.0
    assert a["achieved"] == pytest.approx((1_000_000 * 420 + 250_000 * 96) / 0.005 / 1e9)
    assert a["frac"] == pytest.approx(a["achieved"] / 6000.0)


def test_cpu_baseline_walks_the_handed_over_trees():
    """cpu_equal_work loads a trainer's rows into the oracle and times that
    trainer's next update: the oracle's counters there equal the ones of the
    trainer that produced the rows, run one update further."""
    sys.path.insert(0, str(ROOT))
    import bench as b
    import binding
    from conftest import mccfr

    L = mccfr.lib
    cfg = L.preset(L.PRESET_HU_20BB)
    cfg.table_log2 = 20
    table = mccfr.hand_table()
    src = binding.Oracle(cfg, table)
    src.train(2, 512, threads=2)
    rows = src.export_rows()
    c0 = src.counters()
    src.step(3, 0, 512, threads=2)
    c1 = src.counters()
    out = b.cpu_equal_work(rows, cfg, 2, 512, table, 512)
    assert out["kind"] == "port" and out["value"] > 0 and out["rows_loaded"] == rows["keys"].size
    assert out["V_per_traversal"] == pytest.approx((c1["visits"] - c0["visits"]) / 512)
    assert out["U_per_traversal"] == pytest.approx((c1["updates"] - c0["updates"]) / 512)
    assert "iteration 3, player 0" in out["sample"]
