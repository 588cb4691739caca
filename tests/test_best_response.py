"""Heads-up best response (mccfr_best_response, host FP64) against the
brute-force checker, plus the properties every best response must have.

The strategies evaluated come from the CPU oracle's training, so these tests
need no GPU; the GPU-trained strategies are compared in
test_gpu_exploitability.py."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import mccfr

import binding as B
import br_brute as BB

L = mccfr.lib


def subgame_config(sizes=((1, 2), (1, 1)), table_log2=16) -> L.Config:
    c = L.preset(L.PRESET_HU_20BB)
    c.small_blind, c.big_blind, c.starting_stack = 50, 100, 10000
    slots = [(L.ACT_FOLD, 0, 1), (L.ACT_CHECK_CALL, 0, 1)] + [(L.ACT_RAISE_POT, n, d) for n, d in sizes]
    slots.append((L.ACT_ALL_IN, 0, 1))
    c.num_actions = len(slots)
    for a, (k, n, d) in enumerate(slots):
        c.action_kind[a], c.action_num[a], c.action_den[a] = k, n, d
    c.raise_cap = 2
    c.max_depth = 255
    c.table_log2 = table_log2
    c.key_bits = table_log2 - 1
    return c


def small_subgame(street: int, n_combos: int, seed: int) -> dict:
    rng = np.random.default_rng(seed)
    board = [int(c) for c in rng.permutation(52)[:5]]
    nb = 4 if street == 2 else 5
    ranges = np.zeros((2, 1326), np.float32)
    for p in range(2):
        for c in rng.permutation(1326):
            lo, hi = BB.combo_cards(int(c))
            if lo in board[:nb] or hi in board[:nb]:
                continue
            ranges[p, c] = rng.uniform(0.2, 1.0)
            if (ranges[p] > 0).sum() >= n_combos:
                break
    return dict(street=street, pot=1000, board=board, ranges=ranges)


@pytest.mark.parametrize("street,n_combos,sampling,seed", [
    (3, 6, L.SAMPLING_EXTERNAL, 3), (3, 5, L.SAMPLING_REFERENCE, 4), (2, 3, L.SAMPLING_EXTERNAL, 2),
])
def test_subgame_matches_brute_force(hand_table, street, n_combos, sampling, seed):
    cfg = subgame_config()
    cfg.sampling = sampling
    sg = small_subgame(street, n_combos, seed)
    o = B.Oracle(cfg, hand_table, subgame=sg)
    o.train(20, 256)
    rows = o.export_rows()
    assert rows["keys"].size > 0
    r = L.best_response(cfg, hand_table, rows["keys"], rows["strategy_sum"], subgame=sg, threads=2)
    b = BB.best_response_values(cfg, street, sg["pot"], sg["board"], sg["ranges"], hand_table, rows["keys"],
                                rows["strategy_sum"])
    for p in range(2):
        assert r["br_value"][p] == pytest.approx(b[p], rel=1e-9, abs=1e-9)
        assert r["br_value"][p] >= r["profile_value"][p] - 1e-9
    assert r["profile_value"][0] + r["profile_value"][1] == pytest.approx(0.0, abs=1e-9)
    assert r["exploitability"] >= 0.0
    assert r["mbb_per_game"] == pytest.approx(r["exploitability"] / cfg.big_blind * 1000.0)


def test_subgame_untrained_is_uniform(hand_table):
    """No rows at all: every node plays uniformly; the brute force agrees."""
    cfg = subgame_config(sizes=((1, 1),))
    sg = small_subgame(3, 4, 11)
    keys = np.zeros(0, np.uint64)
    ss = np.zeros((0, 8), np.float32)
    r = L.best_response(cfg, hand_table, keys, ss, subgame=sg)
    b = BB.best_response_values(cfg, 3, sg["pot"], sg["board"], sg["ranges"], hand_table, keys, ss)
    assert r["br_value"][0] == pytest.approx(b[0], rel=1e-9)
    assert r["br_value"][1] == pytest.approx(b[1], rel=1e-9)


def test_rank_cdf_lut_matches_oracle(hand_table):
    for n, buckets in ((5, 50), (6, 200), (7, 50)):
        ours = L.rank_cdf_lut(hand_table, n, buckets)
        ref = np.zeros(7463, np.uint8)
        B.lib().orc_rank_cdf_lut(B._p(hand_table), n, buckets, B._p(ref))
        assert np.array_equal(ours, ref), n


def test_full_game_sampled_flops(hand_table):
    """HU 20BB from the blinds on every 350th flop class: the suit-permutation
    self-check agrees, values are zero-sum, and a best response never loses to
    the profile.  With no rows both seats play the same uniform strategy, so
    both best responses are worth the same."""
    cfg = L.preset(L.PRESET_HU_20BB)
    keys = np.zeros(0, np.uint64)
    ss = np.zeros((0, 8), np.float32)
    r = L.best_response(cfg, hand_table, keys, ss, flop_stride=350, iso_check=True)
    assert not r["exact"]
    assert r["iso_check"] < 1e-12
    assert r["br_value"][0] == pytest.approx(r["br_value"][1], rel=1e-12)
    assert abs(r["profile_value"][0]) < 1e-9 and abs(r["profile_value"][1]) < 1e-9
    assert r["mbb_per_game"] > 1000.0  # uniform play is very exploitable


def test_full_game_trained_strategy_properties(hand_table):
    cfg = L.preset(L.PRESET_HU_20BB)
    cfg.table_log2 = 22
    cfg.key_bits = 21
    o = B.Oracle(cfg, hand_table)
    o.train(1, 2048)
    rows = o.export_rows()
    r = L.best_response(cfg, hand_table, rows["keys"], rows["strategy_sum"], flop_stride=350, iso_check=True)
    assert r["iso_check"] < 1e-12
    assert r["profile_value"][0] + r["profile_value"][1] == pytest.approx(0.0, abs=1e-9)
    for p in range(2):
        assert r["br_value"][p] >= r["profile_value"][p] - 1e-9


def test_rejects_unsupported(hand_table):
    keys = np.zeros(0, np.uint64)
    ss = np.zeros((0, 8), np.float32)
    six = L.preset(L.PRESET_6MAX_100BB)
    with pytest.raises(L.MccfrError):
        L.best_response(six, hand_table, keys, ss)
    ref = L.preset(L.PRESET_REF8)  # rank-linear buckets on chain states: not suit-invariant
    with pytest.raises(L.MccfrError):
        L.best_response(ref, hand_table, keys, ss)
    cfg = subgame_config()
    sg = small_subgame(3, 1, 5)
    sg["ranges"][1] = 0.0
    lo, hi = BB.combo_cards(int(np.flatnonzero(sg["ranges"][0])[0]))
    for c in range(1326):  # only combos that collide with player 0's single combo
        a, b = BB.combo_cards(c)
        if (a in (lo, hi) or b in (lo, hi)) and a not in sg["board"] and b not in sg["board"]:
            sg["ranges"][1][c] = 1.0
    with pytest.raises(L.MccfrError):
        L.best_response(cfg, hand_table, keys, ss, subgame=sg)
