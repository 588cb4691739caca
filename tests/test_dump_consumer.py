"""The v2 strategy dump read and played by the reference's own consumers:
strategy_load_auto / strategy_load (poker_cuda/src/strategy.cpp:54-138) and
evaluate_strategy_np against the scripted archetypes (poker_cuda/src/eval.cpp:
604-627), compiled unchanged into oracle/_ref/libref_eval.so.

CPU: a dump in the product's format from the oracle's training.  GPU: the dump
mccfr_save_strategy writes after training on the device."""
from __future__ import annotations

import numpy as np
import pytest

import binding
from conftest import mccfr

L = mccfr.lib
pytestmark = pytest.mark.skipif(not binding.ref_eval_available(),
                                reason="the reference's sources were not built here")


@pytest.fixture(scope="module")
def ref_eval(hand_table_file):
    r = binding.ref_eval()
    assert r.refeval_init(str(hand_table_file).encode()) == 1
    return r


def playable(probs: np.ndarray) -> np.ndarray:
    """Rows strategy_load keeps: it drops rows that are exactly uniform over
    all eight slots as placeholders of an older export (strategy.cpp:22-33)."""
    return ~np.all(np.abs(probs - 0.125) <= 1e-6, axis=1)


def check_dump(ref_eval, path, keys, probs):
    keep = playable(probs)
    assert ref_eval.refeval_load(str(path).encode()) == int(keep.sum()) > 0
    got = np.zeros(8, np.float32)
    for i in np.flatnonzero(keep)[:: max(1, int(keep.sum()) // 64)]:
        assert ref_eval.refeval_entry(int(keys[i]), binding._p(got)) == 1
        assert np.array_equal(got, probs[i])
    res = {o: binding.ref_play(o, 20000) for o in binding.OPPONENTS}
    for r in res.values():
        assert r["hands"] == 20000 and np.isfinite(r["bb_per_100"])
    assert binding.ref_play("maniac", 20000) == res["maniac"]  # seeded: repeatable
    return res


def test_oracle_dump_plays_in_the_reference(hand_table, ref_eval, tmp_path):
    cfg = L.preset(L.PRESET_REF8)
    o = binding.Oracle(cfg, hand_table)
    o.train(4, 2048)
    keys, probs = o.strategy_arrays()
    dump = tmp_path / "s.bin"
    binding.write_strategy_v2(dump, keys, probs)
    res = check_dump(ref_eval, dump, keys, probs)
    # the bot plays the table: with no rows it falls back to passive play
    empty = tmp_path / "empty.bin"
    binding.write_strategy_v2(empty, np.zeros(0, np.uint32), np.zeros((0, 8), np.float32))
    assert ref_eval.refeval_load(str(empty).encode()) == 0
    assert binding.ref_play("maniac", 20000) != res["maniac"]


@pytest.mark.gpu
def test_device_dump_plays_in_the_reference(hand_table, ref_eval, tmp_path):
    cfg = L.preset(L.PRESET_REF8)
    cfg.table_log2 = 20
    tr = mccfr.GPUCFRTrainer(config=cfg)
    tr.set_hand_table(hand_table)
    tr.train(4, 2048, verbose=False)
    dump = tmp_path / "s.bin"
    assert tr.save_strategy(str(dump))
    keys, probs = tr.strategy_arrays()
    check_dump(ref_eval, dump, keys, probs)
    tr.close()
