"""The batched forms against the plain trainer: every table of a batch ends
bit-identical to the same table trained alone, whatever the tuning and form
(one persistent traversal launch per phase, or every table's own update
kernels as concurrent branches of one graph)."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import mccfr

L = mccfr.lib
pytestmark = pytest.mark.gpu


def small_tables():
    """Three uneven tables: heads-up 20BB, 6-max 100BB, and 3-handed 50BB with 3 actions."""
    hu = L.preset(L.PRESET_HU_20BB)
    six = L.preset(L.PRESET_6MAX_100BB)
    three = L.preset(L.PRESET_HU_20BB)
    three.num_players = 3
    three.starting_stack = 5000
    three.num_actions = 3
    three.action_kind[2] = L.ACT_ALL_IN
    three.seed = 7
    out = []
    for c in (hu, six, three):
        c.table_log2 = 22
        c.key_bits = 21
        out.append(c)
    return out, [3000, 200, 1500]


def make(cfgs, table):
    ts = []
    for c in cfgs:
        t = mccfr.GPUCFRTrainer(config=c)
        t.set_hand_table(table)
        ts.append(t)
    return ts


def rows_equal(a, b):
    for f in ("keys", "visits", "regrets", "strategy_sum"):
        assert np.array_equal(np.asarray(a[f]).view(np.uint8), np.asarray(b[f]).view(np.uint8)), f


def test_batched_equals_plain(hand_table):
    cfgs, trav = small_tables()
    plain = make(cfgs, hand_table)
    for t, n in zip(plain, trav):
        t.train(2, n, verbose=False)
    batched = make(cfgs, hand_table)
    b = mccfr.Batch(batched, trav)
    b.train(2)
    for p, q in zip(plain, batched):
        rows_equal(p.export_rows(), q.export_rows())
    st = b.stats()
    assert st.iterations == 2
    assert st.traversals == sum(2 * n * c.num_players for n, c in zip(trav, cfgs))
    b.close()


def test_autotune_keeps_results(hand_table):
    cfgs, trav = small_tables()
    plain = make(cfgs, hand_table)
    batched = make(cfgs, hand_table)
    b = mccfr.Batch(batched, trav)
    best = b.autotune(max_candidates=6)  # 12 real iterations: the list forward, then backward
    assert best in mccfr.Batch.candidates(6)
    b.set_tuning(block=64, grab=4, smem_frames=2, probe_width=2, warp_sync=0)
    b.train(1)
    for t, n in zip(plain, trav):
        t.train(13, n, verbose=False)
    for p, q in zip(plain, batched):
        rows_equal(p.export_rows(), q.export_rows())
    b.close()


def test_table_graph_form_equals_plain(hand_table):
    """Two iterations in the table-graph form, then one in the persistent form and
    one more in the table-graph form: each table equals four iterations of
    training it alone (the level-synchronous kernels in its branch)."""
    cfgs, trav = small_tables()
    plain = make(cfgs, hand_table)
    for t, n in zip(plain, trav):
        t.train(4, n, verbose=False)
    batched = make(cfgs, hand_table)
    b = mccfr.Batch(batched, trav)
    b.set_tuning(form=L.BATCH_TABLE_GRAPHS)
    b.train(2, timed=True)
    b.set_tuning(form=L.BATCH_PERSISTENT)
    b.train(1)
    b.set_tuning(form=L.BATCH_TABLE_GRAPHS)
    b.train(1)
    for p, q in zip(plain, batched):
        rows_equal(p.export_rows(), q.export_rows())
    st = b.stats()
    assert st.iterations == 4
    assert st.traversals == sum(4 * n * c.num_players for n, c in zip(trav, cfgs))
    assert st.total_ms > 0
    b.close()


def test_a_table_twice_is_refused(hand_table):
    cfgs, trav = small_tables()
    ts = make(cfgs[:1], hand_table)
    with pytest.raises(L.MccfrError):
        mccfr.Batch([ts[0], ts[0]], [trav[0], trav[0]])
    ts[0].close()
