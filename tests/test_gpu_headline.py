"""The 6-max 100BB configuration against the oracle at the shape the benchmark
times: the graph path (`train`), iterations into the benchmark's window, the
full 2^20-traversal update, the batched form, and the FP32 order of the
reference's atomics over many player-updates.

Every traversal form (depth-first lanes and the level-synchronous kernels)
must give the oracle's rows bit for bit; the FP32 comparison states the
tolerance north of it: cumulative regrets and strategy sums within 1e-5
relative (absolute 1e-5 below magnitude 1).
"""
from __future__ import annotations

import os

import numpy as np
import pytest

import binding
from conftest import mccfr

L = mccfr.lib
pytestmark = pytest.mark.gpu

FORMS = [L.FORM_LANES, L.FORM_LEVELS]
FORM_IDS = ["lanes", "levels"]
THREADS = os.cpu_count() or 8


def assert_rows_equal(g, o):
    assert np.array_equal(g["keys"], o["keys"])
    assert np.array_equal(g["visits"], o["visits"])
    assert np.array_equal(g["regrets"].view(np.uint32), o["regrets"].view(np.uint32))
    assert np.array_equal(g["strategy_sum"].view(np.uint32), o["strategy_sum"].view(np.uint32))


def trainer(cfg, table):
    t = mccfr.GPUCFRTrainer(config=cfg)
    t.set_hand_table(table)
    return t


@pytest.mark.parametrize("form", FORMS, ids=FORM_IDS)
def test_graph_training_equals_oracle_every_iteration(hand_table, form):
    """25 iterations of 4,096 traversals per player-update through `train` (one
    graph replay per iteration) on the preset's own 2^27-row direct-mapped
    table: the table digest equals the oracle's after every iteration, and every
    row is compared after iterations 1, 6 and 25.  Trees run from about 630
    decision nodes per traversal (iteration 1) down to about 160."""
    cfg = L.preset(L.PRESET_6MAX_100BB)
    cfg.traversal_form = form
    tr = trainer(cfg, hand_table)
    orc = binding.Oracle(cfg, hand_table)
    for it in range(1, 26):
        tr.train(1, 4096, verbose=False)
        orc.train(1, 4096, threads=THREADS)
        assert tr.digest() == orc.digest(), f"iteration {it}"
        if it in (1, 6, 25):
            assert_rows_equal(tr.export_rows(), orc.export_rows())
    st, oc = tr.stats(), orc.counters()
    assert (st.traversals, st.node_visits, st.traverser_updates, st.terminals) == (
        oc["traversals"], oc["visits"], oc["updates"], oc["terminals"])
    tr.close()
    orc.close()


@pytest.mark.parametrize("form", FORMS, ids=FORM_IDS)
def test_full_size_update_equals_oracle(hand_table, form):
    """The benchmark's own shape: 2^20 traversals per player-update on the
    2^27-row table.  After five device iterations the table (every one of the
    2^26 key values in use) is handed to the oracle; iteration 6, inside the
    benchmark's timed window, then runs on both from the same rows: through the
    training graph on the device, update by update on the oracle."""
    cfg = L.preset(L.PRESET_6MAX_100BB)
    cfg.traversal_form = form
    batch = 1 << 20
    tr = trainer(cfg, hand_table)
    tr.train(5, batch, verbose=False)
    orc = binding.Oracle(cfg, hand_table)
    rows = tr.export_rows()
    assert rows["keys"].size > (1 << 25)
    orc.import_rows(rows, 5)
    del rows
    assert tr.digest() == orc.digest()
    s0 = tr.stats()
    tr.train(1, batch, verbose=False)
    s1 = tr.stats()
    for p in range(6):
        orc.step(6, p, batch, threads=THREADS)
    assert tr.digest() == orc.digest()
    oc = orc.counters()
    assert (s1.node_visits - s0.node_visits, s1.traverser_updates - s0.traverser_updates,
            s1.terminals - s0.terminals) == (oc["visits"], oc["updates"], oc["terminals"])
    assert oc["visits"] > 40 * 6 * batch  # trees of the timed window, not of iteration 1
    tr.close()
    orc.close()


@pytest.mark.parametrize("lg", [8, 14, 16])
def test_level_buffers_smaller_than_the_update(hand_table, lg):
    """The level form with node buffers far below its default of 64 per
    traversal (2^lg node records for 4,096 traversals, and as many showdown
    records): a seed that may not fit is left to the depth-first kernel (at
    lg = 8 every root is, at lg = 14 the levels below the first, at lg = 16
    whatever no longer fits part-way through a level), and a showdown past the
    end of its record list is evaluated where it is reached.  Three iterations
    from an empty table; the table digest equals the oracle's after each, and
    every row after the last."""
    cfg = L.preset(L.PRESET_6MAX_100BB)
    cfg.table_log2, cfg.key_bits = 22, 21
    cfg.traversal_form = L.FORM_LEVELS
    cfg.level_log2 = lg
    tr = trainer(cfg, hand_table)
    orc = binding.Oracle(cfg, hand_table)
    for it in range(1, 4):
        tr.train(1, 4096, verbose=False)
        orc.train(1, 4096, threads=THREADS)
        assert tr.digest() == orc.digest(), f"iteration {it}"
    assert_rows_equal(tr.export_rows(), orc.export_rows())
    lv = tr.level_counts()
    if lg <= 14:
        assert lv["deferred"] > 0
    st, oc = tr.stats(), orc.counters()
    assert (st.node_visits, st.traverser_updates, st.terminals) == (oc["visits"], oc["updates"], oc["terminals"])
    tr.close()
    orc.close()


def uneven_tables():
    """Four tables of different shapes: 2, 3, 4 and 6 players; stacks 20, 50,
    80 and 150BB; 4, 3, 5 and 6 action slots; per-update traversals uneven."""
    specs = []
    for n, bb, na, trav, seed in ((2, 20, 4, 3000, 11), (3, 50, 3, 1500, 12), (4, 80, 5, 700, 13),
                                  (6, 150, 6, 300, 14)):
        c = L.preset(L.PRESET_HU_20BB)
        c.num_players = n
        c.starting_stack = bb * c.big_blind
        slots = {3: [(L.ACT_FOLD, 0, 1), (L.ACT_CHECK_CALL, 0, 1), (L.ACT_ALL_IN, 0, 1)],
                 4: [(L.ACT_FOLD, 0, 1), (L.ACT_CHECK_CALL, 0, 1), (L.ACT_RAISE_POT, 1, 1), (L.ACT_ALL_IN, 0, 1)],
                 5: [(L.ACT_FOLD, 0, 1), (L.ACT_CHECK_CALL, 0, 1), (L.ACT_RAISE_POT, 1, 2), (L.ACT_RAISE_POT, 1, 1),
                     (L.ACT_ALL_IN, 0, 1)],
                 6: [(L.ACT_FOLD, 0, 1), (L.ACT_CHECK_CALL, 0, 1), (L.ACT_RAISE_POT, 1, 2), (L.ACT_RAISE_POT, 1, 1),
                     (L.ACT_RAISE_POT, 2, 1), (L.ACT_ALL_IN, 0, 1)]}[na]
        c.num_actions = na
        for a, (k, num, den) in enumerate(slots):
            c.action_kind[a], c.action_num[a], c.action_den[a] = k, num, den
        c.raise_cap = 3
        c.table_log2 = 22
        c.key_bits = 21
        c.seed = seed
        specs.append((c, trav))
    return specs


def test_batched_form_equals_oracle(hand_table):
    """Four uneven tables in one batch, three iterations: each table's rows
    equal its own oracle's."""
    specs = uneven_tables()
    ts = [trainer(c, hand_table) for c, _ in specs]
    b = mccfr.Batch(ts, [n for _, n in specs])
    b.train(3)
    for (c, n), t in zip(specs, ts):
        orc = binding.Oracle(c, hand_table)
        orc.train(3, n, threads=THREADS)
        assert_rows_equal(t.export_rows(), orc.export_rows())
        orc.close()
    b.close()
    for t in ts:
        t.close()


def fp32_cases():
    six = L.preset(L.PRESET_6MAX_100BB)
    six.table_log2, six.key_bits = 24, 24
    ref6 = L.preset(L.PRESET_REF8)
    ref6.num_players = 6
    ref6.table_log2 = 26
    return [(six, 4096, "6max-100bb external sampling"), (ref6, 8192, "reference game, reference rule, 6 players")]


@pytest.mark.parametrize("case", [0, 1], ids=["6max-es", "ref8-6p"])
def test_fp32_order_within_tolerance_over_updates(hand_table, case):
    """Twelve player-updates (two iterations of six players).  Before each update
    the device's rows are handed to the oracle in FP32 mode, which adds every
    delta as an FP32 value in traversal order (the reference's atomics,
    cfr_gpu.cu:788, 1006-1007) instead of summing exactly in fixed point; after
    the update both tables hold the same keys, and every row's regrets and
    strategy sums agree within 1e-5 of the row's largest magnitude (at least 1):
    |a - b| <= 1e-5 * max(max_row |b|, 1).  The bound is per row because a value
    that is the cancellation of large deltas carries the FP32 order's own
    rounding (about 2^-12 chips for 6-max deltas of thousands of chips), which no
    elementwise relative bound can hold near zero; the elementwise worst case is
    reported beside it."""
    cfg, batch, _ = fp32_cases()[case]
    tr = trainer(cfg, hand_table)
    orc = binding.Oracle(cfg, hand_table)
    orc.set_float_mode(True)
    worst_row, worst_elem = 0.0, 0.0
    for it in (1, 2):
        for p in range(cfg.num_players):
            before = tr.export_rows()
            tr.step(it, p, batch)
            orc.import_rows(before, it - 1)
            orc.step(it, p, batch, threads=1)
            g, o = tr.export_rows(), orc.export_rows()
            assert np.array_equal(g["keys"], o["keys"])
            assert np.array_equal(g["visits"], o["visits"])
            for f in ("regrets", "strategy_sum"):
                a, b = g[f].astype(np.float64), o[f].astype(np.float64)
                if not a.size:
                    continue
                scale = np.maximum(np.abs(b).max(axis=1, keepdims=True), 1.0)
                err = np.abs(a - b) / scale
                worst_row = max(worst_row, float(err.max()))
                worst_elem = max(worst_elem, float((np.abs(a - b) / np.maximum(np.abs(b), 1.0)).max()))
                assert np.all(err <= 1e-5), (it, p, f, float(err.max()))
    print(f"fp32 order: worst per-row relative difference {worst_row:.3g}, elementwise {worst_elem:.3g}")
    assert worst_row > 0.0  # the two summation orders do differ
    tr.close()
    orc.close()
