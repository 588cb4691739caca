"""CUDA path (through the C ABI) against the CPU oracle on the same seeded inputs.

Bit-exact: dealt cards, buckets, sampled actions, payoffs, info-set keys, visit
counts, regrets and strategy sums (both sides sum deltas in fixed point and apply
them with the same IEEE operations).  Against the reference's FP32 arithmetic
(oracle float mode: deltas added as FP32 in traversal order) the tables agree
within 1e-5 relative.
"""
from __future__ import annotations

import numpy as np
import pytest

import binding
from conftest import mccfr

L = mccfr.lib
pytestmark = pytest.mark.gpu


def make_pair(preset, table, table_log2=20, **over):
    cfg = L.preset(preset)
    cfg.table_log2 = table_log2
    for k, v in over.items():
        setattr(cfg, k, v)
    tr = mccfr.GPUCFRTrainer(config=cfg)
    tr.set_hand_table(table)
    orc = binding.Oracle(cfg, table)
    return cfg, tr, orc


def assert_traces_equal(g, o):
    for f in ("hole", "board", "dealer", "hole_bucket", "board_bucket", "n_actions", "n_traverser_nodes"):
        assert np.array_equal(g[f], o[f]), f
    n = np.minimum(g["n_actions"], 40)
    mask = np.arange(40)[None, :] < n[:, None]
    assert np.array_equal(np.where(mask, g["actions"], 0), np.where(mask, o["actions"], 0))
    assert np.array_equal(g["payoff"].view(np.uint32), o["payoff"].view(np.uint32))


def assert_rows_equal(g, o):
    assert np.array_equal(g["keys"], o["keys"])
    assert np.array_equal(g["visits"], o["visits"])
    assert np.array_equal(g["regrets"].view(np.uint32), o["regrets"].view(np.uint32))
    assert np.array_equal(g["strategy_sum"].view(np.uint32), o["strategy_sum"].view(np.uint32))


@pytest.mark.parametrize("players", [2, 6])
def test_reference_rule_bit_exact(hand_table, players):
    cfg, tr, orc = make_pair(L.PRESET_REF8, hand_table, num_players=players)
    batch = 4096
    for it in (1, 2, 3):
        for p in range(players):
            g = tr.step(it, p, batch, trace=True)
            o = orc.step(it, p, batch, trace=True, trace_dtype=L.TRACE_DTYPE)
            assert_traces_equal(g, o)
    assert_rows_equal(tr.export_rows(), orc.export_rows())
    st, oc = tr.stats(), orc.counters()
    assert (st.traversals, st.node_visits, st.traverser_updates) == (oc["traversals"], oc["visits"], oc["updates"])
    gk, gp = tr.strategy_arrays()
    ok, op = orc.strategy_arrays()
    assert np.array_equal(gk, ok) and np.array_equal(gp.view(np.uint32), op.view(np.uint32))


@pytest.mark.parametrize("preset", [L.PRESET_HU_20BB, L.PRESET_6MAX_100BB])
def test_reference_rule_on_capped_presets(hand_table, preset):
    cfg, tr, orc = make_pair(preset, hand_table, sampling=L.SAMPLING_REFERENCE, max_depth=64)
    for it in (1, 2):
        for p in range(cfg.num_players):
            g = tr.step(it, p, 2048, trace=True)
            o = orc.step(it, p, 2048, trace=True, trace_dtype=L.TRACE_DTYPE)
            assert_traces_equal(g, o)
    assert_rows_equal(tr.export_rows(), orc.export_rows())


@pytest.mark.parametrize("preset,batch", [(L.PRESET_HU_20BB, 2048), (L.PRESET_6MAX_100BB, 64)])
def test_external_sampling_bit_exact(hand_table, preset, batch):
    cfg, tr, orc = make_pair(preset, hand_table, table_log2=22)
    for it in (1, 2):
        for p in range(cfg.num_players):
            tr.step(it, p, batch)
            orc.step(it, p, batch)
    assert_rows_equal(tr.export_rows(), orc.export_rows())
    st, oc = tr.stats(), orc.counters()
    assert (st.node_visits, st.traverser_updates, st.terminals) == (oc["visits"], oc["updates"], oc["terminals"])


def test_external_sampling_on_reference_game(hand_table):
    cfg, tr, orc = make_pair(L.PRESET_REF8, hand_table, table_log2=24, sampling=L.SAMPLING_EXTERNAL)
    for it in (1, 2):
        for p in range(2):
            tr.step(it, p, 1024)
            orc.step(it, p, 1024)
    assert_rows_equal(tr.export_rows(), orc.export_rows())


@pytest.mark.parametrize("preset,sampling,batch", [
    (L.PRESET_6MAX_100BB, L.SAMPLING_EXTERNAL, 64),
    (L.PRESET_HU_20BB, L.SAMPLING_EXTERNAL, 2048),
    (L.PRESET_HU_20BB, L.SAMPLING_REFERENCE, 2048),
])
def test_direct_mapped_table_bit_exact(hand_table, preset, sampling, batch):
    """Keys reduced to 21 bits: in a 2^21-row table key k owns row k-1 and no
    lookup probes; a 2^20-row table holding the same keys probes.  Both equal
    the oracle bit for bit."""
    over = dict(key_bits=21, sampling=sampling)
    if sampling == L.SAMPLING_REFERENCE:
        over["max_depth"] = 64
    cfg, direct, orc = make_pair(preset, hand_table, table_log2=21, **over)
    cfg.table_log2 = 20
    probed = mccfr.GPUCFRTrainer(config=cfg)
    probed.set_hand_table(hand_table)
    for it in (1, 2):
        for p in range(cfg.num_players):
            direct.step(it, p, batch)
            probed.step(it, p, batch)
            orc.step(it, p, batch)
    want = orc.export_rows()
    assert_rows_equal(direct.export_rows(), want)
    assert_rows_equal(probed.export_rows(), want)
    assert want["keys"].size < (1 << 20)  # every key fit the probed table (6-max: 56% full)
    assert want["keys"].max() <= (1 << 21)


def test_graph_training_equals_steps(hand_table):
    cfg = L.preset(L.PRESET_REF8)
    cfg.table_log2 = 20
    a = mccfr.GPUCFRTrainer(config=cfg)
    b = mccfr.GPUCFRTrainer(config=cfg)
    a.set_hand_table(hand_table)
    b.set_hand_table(hand_table)
    a.train(2, 2048, verbose=False)
    a.train(1, 2048, verbose=False, timed=True)
    for it in (1, 2, 3):
        for p in range(2):
            b.step(it, p, 2048)
    assert_rows_equal(a.export_rows(), b.export_rows())
    # the timed graph path counts the last update's touched rows like a step does
    sa, sb = a.stats(), b.stats()
    assert sa.touched_last == sb.touched_last > 0
    assert sa.apply_ms > 0.0
    assert a.rows_used() == b.export_rows()["keys"].size >= sa.touched_last


def test_fp32_reference_order_within_tolerance(hand_table):
    """One player-update from empty tables: the same paths are sampled, and the
    fixed-point sums agree with FP32 sums in traversal order within 1e-5."""
    cfg, tr, orc = make_pair(L.PRESET_REF8, hand_table, num_players=6)
    orc.set_float_mode(True)
    for p in range(6):
        tr.step(1, p, 8192)
        orc.step(1, p, 8192, threads=1)
    g, o = tr.export_rows(), orc.export_rows()
    assert np.array_equal(g["keys"], o["keys"])
    for f in ("regrets", "strategy_sum"):
        a, b = g[f].astype(np.float64), o[f].astype(np.float64)
        tol = 1e-5 * np.maximum(np.abs(b), 1.0)
        assert np.all(np.abs(a - b) <= tol), f


def test_eval7_matches_oracle(hand_table):
    cfg = L.preset(L.PRESET_REF8)
    cfg.table_log2 = 12
    tr = mccfr.GPUCFRTrainer(config=cfg)
    tr.set_hand_table(hand_table)
    rng = np.random.default_rng(3)
    cards = np.argsort(rng.random((1 << 18, 52)), axis=1)[:, :7].astype(np.uint8)
    assert np.array_equal(tr.eval7(cards), binding.eval7(hand_table, cards))


def test_eval7_exhaustive_sweep(hand_table):
    """All C(52, 7) = 133,784,560 hands ranked on the device (mccfr_eval7_device),
    in lexicographic order grouped by the two lowest cards (a, b): each group's
    sum and position-weighted sum of ranks equal the oracle's, so no hand of the
    sweep is missing, misranked or out of order."""
    import ctypes
    import itertools

    import torch

    cfg = L.preset(L.PRESET_REF8)
    cfg.table_log2 = 12
    tr = mccfr.GPUCFRTrainer(config=cfg)
    tr.set_hand_table(hand_table)
    lib = L.load()
    want_s = np.zeros(52 * 52, np.uint64)
    want_w = np.zeros(52 * 52, np.uint64)
    binding.lib().orc_rank7_digests(binding._p(hand_table), binding._p(want_s), binding._p(want_w))
    dev = torch.device("cuda:0")
    # the 5-card completions: combinations of 0..49 in lexicographic order; those
    # below m, shifted by b + 1, are the completions of cards above b
    c5 = torch.from_numpy(np.array(list(itertools.combinations(range(50), 5)), np.uint8)).to(dev)
    got_s = torch.zeros(52 * 52, dtype=torch.int64, device=dev)
    got_w = torch.zeros(52 * 52, dtype=torch.int64, device=dev)
    hands = 0
    for b in range(1, 47):
        tail = c5[c5[:, 4] < 51 - b] + (b + 1)  # cards b+1 .. 51
        n = tail.shape[0]
        pos = torch.arange(1, n + 1, dtype=torch.int64, device=dev)
        cards = torch.empty((n, 7), dtype=torch.uint8, device=dev)
        cards[:, 2:] = tail
        ranks = torch.empty(n, dtype=torch.int16, device=dev)
        for a in range(b):
            cards[:, 0] = a
            cards[:, 1] = b
            torch.cuda.synchronize()  # the library evaluates on its own stream
            L.check(lib.mccfr_eval7_device(tr.handle, ctypes.c_void_p(cards.data_ptr()),
                                           ctypes.c_void_p(ranks.data_ptr()), n, None))
            r = ranks.to(torch.int64) & 0xFFFF
            got_s[a * 52 + b] = r.sum()
            got_w[a * 52 + b] = (r * pos).sum()
            hands += n
    torch.cuda.synchronize()
    assert hands == 133784560
    assert np.array_equal(got_s.cpu().numpy().astype(np.uint64), want_s)
    assert np.array_equal(got_w.cpu().numpy().astype(np.uint64), want_w)
    tr.close()


def test_checkpoint_and_dump_roundtrip(hand_table, tmp_path):
    cfg = L.preset(L.PRESET_REF8)
    cfg.table_log2 = 20
    a = mccfr.GPUCFRTrainer(config=cfg)
    a.set_hand_table(hand_table)
    a.train(2, 4096, verbose=False)
    ck = tmp_path / "s.ckpt"
    assert a.save_checkpoint(str(ck))
    assert ck.stat().st_size == 16 + 2 * 8 * (1 << 26) * 4
    b = mccfr.GPUCFRTrainer(config=cfg)
    b.set_hand_table(hand_table)
    assert b.load_checkpoint(str(ck))
    ra, rb = a.export_rows(), b.export_rows()
    live = (np.abs(ra["regrets"]).sum(1) + np.abs(ra["strategy_sum"]).sum(1)) > 0
    assert np.array_equal(ra["keys"][live], rb["keys"])
    assert np.array_equal(ra["regrets"][live], rb["regrets"])
    assert np.array_equal(ra["strategy_sum"][live], rb["strategy_sum"])
    dump = tmp_path / "s.bin"
    assert a.save_strategy(str(dump))
    raw = dump.read_bytes()
    magic, ts, na, n = np.frombuffer(raw[:8], np.uint64)[0], *np.frombuffer(raw[8:20], np.uint32)
    assert (magic, ts, na) == (0x53545241540100, 1 << 26, 8)
    rec = np.frombuffer(raw[20:], dtype=np.dtype([("k", np.uint32), ("p", np.float32, 8)]))
    keys, probs = a.strategy_arrays()
    assert n == len(rec) == len(keys)
    assert np.array_equal(rec["k"], keys) and np.array_equal(rec["p"], probs)


def test_full_size_properties(hand_table):
    """6-max 100BB at its configured sizes (2^26 hashed keys in a 2^27-row table,
    2^20 traversals per player-update): determinism, a checksum of visit counts,
    CFR+ invariants, normalised strategies."""
    rows = []
    for _ in range(2):
        cfg = L.preset(L.PRESET_6MAX_100BB)
        tr = mccfr.GPUCFRTrainer(config=cfg)
        tr.set_hand_table(hand_table)
        tr.step(1, 0, 1 << 20)
        r = tr.export_rows()
        st = tr.stats()
        assert int(r["visits"].sum()) == st.node_visits  # every decision node updates one row
        assert st.traversals == 1 << 20
        assert np.all(r["regrets"] >= 0) and np.all(r["strategy_sum"] >= 0)
        keys, probs = tr.strategy_arrays()
        assert np.allclose(probs.sum(1), 1.0, atol=1e-5)
        rows.append(r)
        tr.close()
    assert_rows_equal(rows[0], rows[1])
