"""Subgame re-solves and continuous batching on the GPU.

* A subgame trained on the device equals the CPU oracle bit for bit, one
  player-update at a time (mccfr_step) and through the round API.
* Each request served in a mix of concurrent requests (continuous batching,
  admission by device memory) ends with exactly the strategy it gets when it is
  served alone."""
from __future__ import annotations

import numpy as np
import pytest

import binding
from conftest import mccfr

L = mccfr.lib
S = mccfr.serving if hasattr(mccfr, "serving") else None
pytestmark = pytest.mark.gpu


def serving():
    import importlib
    return importlib.import_module("mccfr_b200.serving")


def small_request(rid, street, players, budget=600, seed=5):
    sv = serving()
    rng = np.random.default_rng(seed + rid)
    req = sv.make_request(rng, rid)
    req.street = street
    req.players = players
    req.board = [int(c) for c in rng.permutation(52)[: (4 if street == 2 else 5)]]
    blocked = np.isin(sv.COMBO_CARDS, req.board).any(axis=1)
    r = rng.dirichlet(np.full(1326, 0.5), size=players)
    r[:, blocked] = 0
    req.ranges = (r / r.sum(1, keepdims=True)).astype(np.float32)
    req.pot = 1200 * players
    req.budget = budget
    req.table_log2 = 18
    return req


def rows_equal(a, b):
    for f in ("keys", "visits", "regrets", "strategy_sum"):
        assert np.array_equal(np.asarray(a[f]).view(np.uint8), np.asarray(b[f]).view(np.uint8)), f


@pytest.mark.parametrize("street,players", [(3, 3), (2, 2), (2, 5)])
def test_subgame_matches_oracle(hand_table, street, players):
    sv = serving()
    req = small_request(1, street, players)
    cfg = sv.request_config(req)
    tr = mccfr.GPUCFRTrainer.subgame(cfg, req.street, req.pot, req.board, req.ranges)
    owner = mccfr.GPUCFRTrainer(config=L.preset(L.PRESET_HU_20BB), table_log2=10)
    owner.set_hand_table(hand_table)
    tr.share_hand_table(owner)
    orc = binding.Oracle(cfg, hand_table,
                         subgame={"street": req.street, "pot": req.pot, "board": req.board, "ranges": req.ranges})
    for it in (1, 2):
        for p in range(players):
            tr.step(it, p, 512)
            orc.step(it, p, 512)
    rows_equal(tr.export_rows(), orc.export_rows())
    # the round API continues the same schedule
    tr2 = mccfr.GPUCFRTrainer.subgame(cfg, req.street, req.pot, req.board, req.ranges)
    tr2.share_hand_table(owner)
    for _ in range(2 * players):
        mccfr.batch_round([tr2], [512])
    assert tr2.progress() == (3, 0, 2)
    rows_equal(tr2.export_rows(), orc.export_rows())


def test_each_request_same_alone_and_mixed(hand_table):
    sv = serving()
    owner = mccfr.GPUCFRTrainer(config=L.preset(L.PRESET_HU_20BB), table_log2=10)
    owner.set_hand_table(hand_table)
    reqs = [small_request(i, 2 + (i % 2), 2 + (i % 5), budget=300 + 150 * i) for i in range(6)]
    # mixed: a budget that holds only 3 tables at a time, so admissions interleave
    mixed = sv.ReSolveServer(owner, hbm_budget=3 * sv.table_bytes(reqs[0]) + 1, traversals=128)
    out = {r.rid: r for r in mixed.run(reqs, realtime=False)}
    assert len(out) == len(reqs)
    for req in reqs:
        alone = sv.ReSolveServer(owner, traversals=128).run([req], realtime=False)[0]
        assert np.array_equal(alone.keys, out[req.rid].keys)
        assert np.array_equal(alone.probs.view(np.uint32), out[req.rid].probs.view(np.uint32))


def test_reset_table_equals_fresh_table(hand_table):
    """A subgame trainer reset to another subgame (mccfr_subgame_reset) trains
    exactly like a trainer created for that subgame."""
    sv = serving()
    owner = mccfr.GPUCFRTrainer(config=L.preset(L.PRESET_HU_20BB), table_log2=10)
    owner.set_hand_table(hand_table)
    a = small_request(11, 3, 4)
    b = small_request(12, 2, 3)
    b.table_log2 = a.table_log2
    ca, cb = sv.request_config(a), sv.request_config(b)
    reused = mccfr.GPUCFRTrainer.subgame(ca, a.street, a.pot, a.board, a.ranges)
    reused.share_hand_table(owner)
    reused.train(2, 512, verbose=False)
    reused.reset_subgame(cb, b.street, b.pot, b.board, b.ranges)
    fresh = mccfr.GPUCFRTrainer.subgame(cb, b.street, b.pot, b.board, b.ranges)
    fresh.share_hand_table(owner)
    for t in (reused, fresh):
        t.train(2, 512, verbose=False)
        mccfr.batch_round([t], [256])
    rows_equal(reused.export_rows(), fresh.export_rows())
    assert reused.progress() == fresh.progress()
    for t in (reused, fresh, owner):
        t.close()
