"""The oracle's restatements against the reference's own functions and against
published known answers (CPU)."""
from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np
import pytest

import binding
from conftest import mccfr

L = mccfr.lib
PINS = Path(__file__).parent / "golden" / "ref_pins.npz"


def test_philox_known_answers():
    """Philox4x32-10 known-answer vectors of the Random123 distribution
    (Salmon et al., SC'11)."""
    kat = [
        ((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
        ((0xFFFFFFFF,) * 4, (0xFFFFFFFF,) * 2, (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
        ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
         (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
    ]
    for ctr, key, want in kat:
        assert tuple(int(x) for x in binding.philox(ctr, key)) == want


def test_uniform_mapping():
    u = binding.lib().orc_uniform01
    assert u(0) == 2.0 ** -24
    assert u(0xFFFFFFFF) == 1.0
    assert u(0x80000000) == (2 ** 23 + 1) * 2.0 ** -24


def test_preflop_buckets_match_reference():
    pins = np.load(PINS)
    lut = binding.preflop_lut(L.PREFLOP_CHEN64, 64).reshape(52, 52)
    assert np.array_equal(lut, pins["pre"])
    c169 = binding.preflop_lut(L.PREFLOP_CLASS169, 169).reshape(52, 52)
    ids = {int(c169[a, b]) for a in range(52) for b in range(52) if a != b}
    assert ids == set(range(169))


def test_action_rules_match_reference():
    pins = np.load(PINS)
    cfg = L.preset(L.PRESET_REF8)
    for s, m, ch in zip(pins["states"], pins["masks"], pins["chips"]):
        pot, stack, to_call, cb, lfr, bb = map(int, s)
        cfg.big_blind = bb
        assert binding.valid_mask(cfg, pot, stack, to_call, cb, lfr) == int(m)
        for a in range(8):
            assert binding.chips(cfg, a, pot, stack, to_call, cb, lfr) == int(ch[a])


def test_postflop_buckets_follow_gpu_rule(hand_table):
    """The reference's GPU bucket (cfr_gpu.cu:487-488) truncates to 8 bits while
    its CPU twin (abstraction.cpp:71-72) clamps at 127: they agree whenever the
    unclamped value is below 127, and the oracle follows the GPU."""
    pins = np.load(PINS)
    cards = pins["cards"]
    lib = binding.lib()
    agree = 0
    for i in range(cards.shape[0]):
        h0, h1 = int(cards[i, 0]), int(cards[i, 1])
        comm = np.ascontiguousarray(cards[i, 2:])
        for st in (1, 2, 3):
            o = lib.orc_ref_board_bucket(L.ptr(hand_table), h0, h1, L.ptr(comm), st, 128)
            cpu = int(pins["fast"][i, st - 1])
            if cpu < 127:
                assert o == cpu
                agree += 1
    assert agree > 0.4 * 3 * cards.shape[0]


def test_rank_cdf_buckets_are_monotone(hand_table):
    for n, b in ((5, 50), (6, 200), (7, 200)):
        out = np.zeros(7463, dtype=np.uint8)
        binding.lib().orc_rank_cdf_lut(L.ptr(hand_table), n, b, L.ptr(out))
        assert np.all(np.diff(out[1:].astype(int)) >= 0)
        assert out[1] == 0 and out[7462] == b - 1


def test_regret_fraction_bits():
    cfg = L.preset(L.PRESET_6MAX_100BB)
    rb = binding.lib().orc_regret_frac_bits(ctypes.byref(cfg), 1 << 20)
    # batch * 64 visits * 20 * N * stack * 2^rb must stay below 2^61
    assert 8 <= rb <= 24
    assert (1 << 20) * 64 * 20 * 6 * 10000 * (1 << rb) < (1 << 63)


def test_thread_count_does_not_change_rows(hand_table):
    """The oracle sums each update's deltas in integers and folds rows shard by
    shard, so its rows are the same on one thread and on eight."""
    L = mccfr.lib
    for preset, batch, players in ((L.PRESET_6MAX_100BB, 64, 6), (L.PRESET_REF8, 2048, 2)):
        cfg = L.preset(preset)
        rows = []
        for threads in (1, 8):
            o = binding.Oracle(cfg, hand_table)
            for it in (1, 2):
                for p in range(players):
                    o.step(it, p, batch, threads=threads)
            rows.append(o.export_rows())
            o.close()
        for f in ("keys", "visits", "regrets", "strategy_sum"):
            assert np.array_equal(np.asarray(rows[0][f]).view(np.uint8), np.asarray(rows[1][f]).view(np.uint8)), f
        assert rows[0]["keys"].size > 0


def test_showdown_masks_match_the_dealt_hands(hand_table):
    """orc_showdown_masks (the checker for a 6-seat showdown microbench) equals
    winners recomputed from the dealt cards that a traced update records, and
    the seats win evenly."""
    L = mccfr.lib
    cfg = L.preset(L.PRESET_6MAX_100BB)
    cfg.sampling, cfg.max_depth = L.SAMPLING_REFERENCE, 64  # traces exist for the reference rule
    o = binding.Oracle(cfg, hand_table)
    n = 4096
    masks = o.showdown_masks(1, 0, n)
    tr = o.step(1, 0, n, trace=True, trace_dtype=L.TRACE_DTYPE)  # the same deals
    cards = np.concatenate([tr["hole"].reshape(n, 6, 2), np.repeat(tr["board"][:, None, :], 6, axis=1)], axis=2)
    ranks = binding.eval7(hand_table, cards.reshape(-1, 7).astype(np.uint8)).reshape(n, 6)
    want = ((ranks == ranks.max(axis=1, keepdims=True)) * (1 << np.arange(6))).sum(axis=1)
    assert np.array_equal(masks, want.astype(np.uint8))
    big = o.showdown_masks(2, 3, 60000)
    assert np.all((big > 0) & (big < 64))
    wins = np.array([((big >> q) & 1).sum() for q in range(6)])
    expect = wins.mean()
    assert np.all(np.abs(wins - expect) < 5 * np.sqrt(expect))
    split = np.mean([bin(int(x)).count("1") > 1 for x in big])
    assert 0.0 < split < 0.2
    o.close()


def test_oracle_presets_and_table_equal_the_product(hand_table):
    """The oracle's own presets and rank-table generator (used where no device
    library is loaded) give byte-identical configs and the same table."""
    L = mccfr.lib
    for p in (L.PRESET_REF8, L.PRESET_HU_20BB, L.PRESET_6MAX_100BB):
        assert bytes(binding.config_init(L.Config(), p)) == bytes(L.preset(p))
    assert np.array_equal(binding.hand_table(), hand_table)


def test_row_import_continues_training_and_digest(hand_table):
    """Rows handed from one oracle to another (import_rows) continue training
    exactly as the first, and the order-independent digest follows the rows."""
    L = mccfr.lib
    cfg = L.preset(L.PRESET_6MAX_100BB)
    cfg.table_log2, cfg.key_bits = 20, 20
    a = binding.Oracle(cfg, hand_table)
    a.train(1, 128, threads=4)
    b = binding.Oracle(cfg, hand_table)
    b.import_rows(a.export_rows(), 1)
    assert a.digest() == b.digest() and a.digest()[1] == a.export_rows()["keys"].size
    for p in range(6):
        a.step(2, p, 128, threads=4)
        b.step(2, p, 128, threads=1)
    ra, rb = a.export_rows(), b.export_rows()
    for f in ("keys", "visits", "regrets", "strategy_sum"):
        assert np.array_equal(np.asarray(ra[f]).view(np.uint8), np.asarray(rb[f]).view(np.uint8)), f
    assert a.digest() == b.digest()
    c = binding.Oracle(cfg, hand_table)
    assert c.digest() == (0, 0)
    rows = a.export_rows()
    rows["regrets"][0, 0] = np.nextafter(rows["regrets"][0, 0], np.float32(1e9))
    c.import_rows(rows, 2)
    assert c.digest()[0] != a.digest()[0]  # one ulp of one row changes it
    with pytest.raises(ValueError):
        bad = dict(rows)
        bad["keys"] = rows["keys"].copy()
        bad["keys"][0] = 0
        c.import_rows(bad, 2)
