"""The level-synchronous form of a player-update (orc_step_wave) against the
depth-first walk (orc_step): the traversals are expanded one tree level at a
time and their values returned level by level, the shape a breadth-first device
traversal would take.  The rows and counters must be the same bit for bit."""
from __future__ import annotations

import numpy as np
import pytest

import binding
from conftest import mccfr
from test_best_response import subgame_config
from test_gpu_exploitability import river_subgame

L = mccfr.lib


def rows_equal(a, b):
    for f in ("keys", "visits", "regrets", "strategy_sum"):
        assert np.array_equal(np.asarray(a[f]).view(np.uint8), np.asarray(b[f]).view(np.uint8)), f


def both(cfg, hand_table, sched, subgame=None):
    """Runs the schedule both ways; returns the two oracles and the wave
    oracle's counters before its last update."""
    dfs = binding.Oracle(cfg, hand_table, subgame=subgame)
    wave = binding.Oracle(cfg, hand_table, subgame=subgame)
    before = None
    for it, p, batch in sched:
        dfs.step(it, p, batch)
        before = wave.counters()
        assert wave.step_wave(it, p, batch) == 0
    return dfs, wave, before


@pytest.mark.parametrize("name", ["hu-external", "6max-external", "ref8-2p", "ref8-6p", "river-subgame"])
def test_wave_equals_depth_first(hand_table, name):
    sub = None
    if name == "hu-external":
        cfg = L.preset(L.PRESET_HU_20BB)
        sched = [(it, p, 1024) for it in (1, 2, 3) for p in range(2)]
    elif name == "6max-external":
        cfg = L.preset(L.PRESET_6MAX_100BB)
        sched = [(it, p, 48) for it in (1, 2) for p in range(6)]
    elif name == "ref8-2p":
        cfg = L.preset(L.PRESET_REF8)
        sched = [(it, p, 2048) for it in (1, 2, 3) for p in range(2)]
    elif name == "ref8-6p":
        cfg = L.preset(L.PRESET_REF8)
        cfg.num_players = 6
        sched = [(it, p, 1024) for it in (1, 2) for p in range(6)]
    else:
        cfg = subgame_config(table_log2=18)
        sub = river_subgame(9, 60)
        sched = [(it, p, 1024) for it in (1, 2, 3) for p in range(2)]
    dfs, wave, before = both(cfg, hand_table, sched, sub)
    rows_equal(dfs.export_rows(), wave.export_rows())
    assert dfs.counters() == wave.counters()
    # the last update's nodes by depth: one root per traversal; every node is a
    # decision, a terminal or a street change
    hist = wave.wave_hist()
    c = wave.counters()
    assert hist[0] == sched[-1][2]
    decisions = c["visits"] - before["visits"]
    terminals = c["terminals"] - before["terminals"]
    assert decisions + terminals <= hist.sum() <= decisions + terminals + 3 * sched[-1][2] * 64
    dfs.close()
    wave.close()


def test_wave_refuses_float_mode(hand_table):
    o = binding.Oracle(L.preset(L.PRESET_REF8), hand_table)
    o.set_float_mode(True)
    assert o.step_wave(1, 0, 64) == 1
    o.close()
