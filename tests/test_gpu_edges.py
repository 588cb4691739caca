"""Edge cases through the C ABI on the GPU: ragged and single-traversal
batches, empty tables and inputs, invalid cards, and a table that fills up.
Every error here is raised by a host check or by a kernel's own bounds check
(a sticky flag read after the launch)."""
from __future__ import annotations

import numpy as np
import pytest

import binding
from conftest import mccfr

L = mccfr.lib
pytestmark = pytest.mark.gpu

ERR_INVALID_ARG = 1
ERR_TABLE_FULL = 7


def pair(preset, hand_table, **over):
    cfg = L.preset(preset)
    cfg.table_log2 = 20
    for k, v in over.items():
        setattr(cfg, k, v)
    tr = mccfr.GPUCFRTrainer(config=cfg)
    tr.set_hand_table(hand_table)
    return cfg, tr, binding.Oracle(cfg, hand_table)


def rows_equal(g, o):
    for f in ("keys", "visits", "regrets", "strategy_sum"):
        assert np.array_equal(np.asarray(g[f]).view(np.uint8), np.asarray(o[f]).view(np.uint8)), f


@pytest.mark.parametrize("preset,sampling", [
    (L.PRESET_6MAX_100BB, L.SAMPLING_EXTERNAL),
    (L.PRESET_HU_20BB, L.SAMPLING_EXTERNAL),
    (L.PRESET_REF8, L.SAMPLING_REFERENCE),
])
def test_ragged_batches_bit_exact(hand_table, preset, sampling):
    """Batch sizes around the 128-thread block and the 32-lane warp, down to a
    single traversal, with the persistent kernel's work counter handing out
    fewer traversals than it has lanes."""
    over = dict(sampling=sampling)
    if preset != L.PRESET_REF8:
        over["key_bits"] = 19
    cfg, tr, orc = pair(preset, hand_table, **over)
    it = 0
    for batch in (1, 3, 31, 33, 127, 129, 1000):
        it += 1
        for p in range(cfg.num_players):
            tr.step(it, p, batch)
            orc.step(it, p, batch)
    rows_equal(tr.export_rows(), orc.export_rows())
    st, oc = tr.stats(), orc.counters()
    assert st.traversals == oc["traversals"] == cfg.num_players * (1 + 3 + 31 + 33 + 127 + 129 + 1000)
    tr.close()


def test_empty_table_and_zero_iterations(hand_table, tmp_path):
    cfg = L.preset(L.PRESET_HU_20BB)
    cfg.table_log2 = 12
    cfg.key_bits = 11
    tr = mccfr.GPUCFRTrainer(config=cfg)
    tr.set_hand_table(hand_table)
    tr.train(0, 1024, verbose=False)  # no iterations: nothing runs
    assert tr.stats().traversals == 0
    assert tr.rows_used() == 0
    rows = tr.export_rows()
    assert rows["keys"].size == 0 and rows["regrets"].shape[0] == 0
    keys, probs = tr.strategy_arrays()
    assert keys.size == 0 and probs.shape[0] == 0
    assert tr.get_strategy() == {}
    assert tr.num_info_sets_active() == 0
    tr.close()


def test_eval7_empty_single_and_invalid(hand_table):
    cfg = L.preset(L.PRESET_REF8)
    cfg.table_log2 = 12
    tr = mccfr.GPUCFRTrainer(config=cfg)
    tr.set_hand_table(hand_table)
    assert tr.eval7(np.zeros((0, 7), np.uint8)).size == 0
    royal = np.array([[51, 50, 49, 48, 47, 0, 14]], np.uint8)  # As Ks Qs Js Ts 2c 3d
    assert tr.eval7(royal)[0] == 7462
    bad = royal.copy()
    bad[0, 3] = 52  # rejected on the host before any launch
    with pytest.raises(L.MccfrError) as e:
        tr.eval7(bad)
    assert e.value.status == ERR_INVALID_ARG
    tr.close()


def test_table_full_is_reported(hand_table):
    """Full 64-bit keys in a 1024-row probed table: inserts beyond the capacity
    fail their bounded probe, the kernel raises its flag, and the step returns
    MCCFR_ERR_TABLE_FULL instead of faulting."""
    cfg = L.preset(L.PRESET_HU_20BB)
    cfg.table_log2 = 10
    cfg.key_bits = 0
    tr = mccfr.GPUCFRTrainer(config=cfg)
    tr.set_hand_table(hand_table)
    with pytest.raises(L.MccfrError) as e:
        tr.step(1, 0, 2048)
    assert e.value.status == ERR_TABLE_FULL
    tr.close()


def test_train_writes_metrics_lines(hand_table, tmp_path):
    import json

    cfg = L.preset(L.PRESET_HU_20BB)
    cfg.table_log2, cfg.key_bits = 20, 19
    tr = mccfr.GPUCFRTrainer(config=cfg)
    tr.set_hand_table(hand_table)
    log = tmp_path / "metrics.jsonl"
    tr.train(2, 1024, verbose=False, metrics=str(log))
    tr.train(1, 1024, verbose=False, metrics=str(log))
    lines = [json.loads(x) for x in log.read_text().splitlines()]
    assert [m["iteration"] for m in lines] == [2, 3]
    assert [m["traversals"] for m in lines] == [2 * 2 * 1024, 2 * 1024]
    for m in lines:
        assert m["traverse_ms_per_update"] > 0 and m["traversals_per_s"] > 0 and m["device_error"] == 0
    tr.close()
