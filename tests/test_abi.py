"""The C-ABI library loads, exports every declared symbol, and its structs match
the bindings (CPU; no compute calls)."""
from __future__ import annotations

import ctypes
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

from conftest import ROOT, gpu_available, mccfr

L = mccfr.lib
HEADER = ROOT / "include" / "mccfr.h"


def declared_functions() -> set[str]:
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return set(re.findall(r"\b(mccfr_[a-z0-9_]+)\s*\(", text))


def test_every_declared_symbol_is_exported():
    names = declared_functions()
    assert len(names) >= 25
    out = subprocess.run(["nm", "-D", "--defined-only", str(L.LIB_PATH)], capture_output=True, text=True,
                         check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    missing = names - exported
    assert not missing, missing
    lib = L.load()
    for n in names:
        assert getattr(lib, n) is not None
    assert set(L.SIGNATURES) == names


def test_struct_sizes_match():
    sizes = (ctypes.c_size_t * 3)()
    assert L.load().mccfr_abi_sizes(sizes) == 0
    assert sizes[0] == ctypes.sizeof(L.Config)
    assert sizes[1] == ctypes.sizeof(L.Stats)
    assert sizes[2] == ctypes.sizeof(L.Trace) == L.TRACE_DTYPE.itemsize


def test_presets():
    ref8 = L.preset(L.PRESET_REF8)
    assert (ref8.num_players, ref8.starting_stack, ref8.small_blind, ref8.big_blind) == (2, 1000, 10, 20)
    assert ref8.num_actions == 8 and ref8.max_depth == 20 and ref8.seed == 42
    assert ref8.key_mode == L.KEY_FNV26 and ref8.table_log2 == 26  # one row per FNV slot
    assert list(ref8.action_kind) == [0, 1, 2, 4, 5, 5, 5, 6]
    hu = L.preset(L.PRESET_HU_20BB)
    assert hu.num_players == 2 and hu.starting_stack == 20 * hu.big_blind and hu.raise_cap == 2
    assert hu.num_actions == 4 and list(hu.postflop_buckets) == [50, 50, 50] and hu.seed == 0
    six = L.preset(L.PRESET_6MAX_100BB)
    assert six.num_players == 6 and six.starting_stack == 100 * six.big_blind and six.raise_cap == 3
    assert six.num_actions == 6 and list(six.postflop_buckets) == [200, 200, 200] and six.seed == 1
    assert six.table_log2 == 27 and six.key_bits == 26 and six.preflop_buckets == 169
    assert [(six.action_num[a], six.action_den[a]) for a in (2, 3, 4)] == [(1, 2), (1, 1), (2, 1)]
    assert L.load().mccfr_config_init(ctypes.byref(L.Config()), 99) == 1


def test_error_strings_and_invalid_args():
    lib = L.load()
    assert lib.mccfr_strerror(0) == b"ok"
    assert lib.mccfr_strerror(7) == b"info-set table full"
    h = ctypes.c_void_p()
    bad = L.preset(L.PRESET_REF8)
    bad.num_players = 7
    assert lib.mccfr_create(ctypes.byref(bad), ctypes.byref(h)) == 1
    bad = L.preset(L.PRESET_REF8)
    bad.action_kind[0] = 2  # no fold slot left
    assert lib.mccfr_create(ctypes.byref(bad), ctypes.byref(h)) == 1
    assert lib.mccfr_hand_table_generate(None, 10) == 1
    t = np.zeros(10, dtype=np.int32)
    assert lib.mccfr_hand_table_generate(L.ptr(t), 10) == 2


def test_create_without_gpu_fails_cleanly():
    if gpu_available():
        return
    h = ctypes.c_void_p()
    cfg = L.preset(L.PRESET_REF8)
    assert L.load().mccfr_create(ctypes.byref(cfg), ctypes.byref(h)) == L.ERR_NO_DEVICE
    try:
        mccfr.GPUCFRTrainer()
    except mccfr.MccfrError as e:
        assert e.status == L.ERR_NO_DEVICE
    else:
        raise AssertionError("expected MccfrError")


def test_config_validation_without_device():
    for p in (L.PRESET_REF8, L.PRESET_HU_20BB, L.PRESET_6MAX_100BB):
        assert L.validate(L.preset(p)) is None
    cases = [
        (lambda c: setattr(c, "num_players", 7), "players"),
        (lambda c: setattr(c, "table_log2", 9), "table_log2"),
        (lambda c: setattr(c, "key_bits", 60), "key_bits"),
        (lambda c: setattr(c, "max_depth", 0), "max_depth"),
    ]
    for mutate, word in cases:
        c = L.preset(L.PRESET_HU_20BB)
        mutate(c)
        why = L.validate(c)
        assert why is not None and word in why, (word, why)
    c = L.preset(L.PRESET_HU_20BB)
    c.action_kind[0] = L.ACT_CALL  # no fold slot left
    assert "fold" in L.validate(c)



def test_metrics_line_from_stats_snapshots():
    import importlib
    from types import SimpleNamespace

    tm = importlib.import_module("mccfr_b200.trainer")
    s0 = SimpleNamespace(traversals=100, node_visits=1000, traverser_updates=200, hand_evals=300, launches=6,
                         traverse_ms=10.0, apply_ms=2.0, iterations_done=1, touched_last=5, device_error=0)
    s1 = SimpleNamespace(traversals=2100, node_visits=101000, traverser_updates=20200, hand_evals=4300,
                         launches=10, traverse_ms=30.0, apply_ms=6.0, iterations_done=3, touched_last=77,
                         device_error=0)
    m = tm.metrics_line(s0, s1, 2.0, 2, 1000)
    assert m["iteration"] == 3 and m["traversals"] == 2000 and m["traversals_per_s"] == 1000.0
    assert m["node_visits_per_s"] == 50000.0 and m["hand_evals_per_s"] == 2000.0
    assert m["traverse_ms_per_update"] == 5.0 and m["apply_ms_per_update"] == 1.0
    assert m["algorithmic_gbs"] == pytest.approx((40 * 100000 + 96 * 20000) / 0.020 / 1e9)
    assert m["touched_rows_last_update"] == 77
