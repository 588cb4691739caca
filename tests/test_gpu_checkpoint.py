"""Checkpoint v2 (mccfr_save/load_checkpoint_v2): training resumed from the file
equals uninterrupted training bit for bit, in direct-mapped and probed tables;
files for another game, truncated files and keys outside the table are refused
on the host before anything reaches the device."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from conftest import mccfr

L = mccfr.lib
pytestmark = pytest.mark.gpu

ERR_INVALID_ARG = 1
ERR_FORMAT = 5


def rows_equal(g, o):
    for f in ("keys", "visits", "regrets", "strategy_sum"):
        assert np.array_equal(np.asarray(g[f]).view(np.uint8), np.asarray(o[f]).view(np.uint8)), f


def trainer(cfg, hand_table):
    t = mccfr.GPUCFRTrainer(config=L.Config.from_buffer_copy(cfg))
    t.set_hand_table(hand_table)
    return t


@pytest.mark.parametrize("key_bits,table_log2", [(19, 20), (22, 20)], ids=["direct", "probed"])
def test_resume_equals_uninterrupted(hand_table, tmp_path, key_bits, table_log2):
    cfg = L.preset(L.PRESET_HU_20BB)
    cfg.table_log2, cfg.key_bits = table_log2, key_bits
    straight = trainer(cfg, hand_table)
    straight.train(5, 2048, verbose=False)
    a = trainer(cfg, hand_table)
    a.train(3, 2048, verbose=False)
    ck = tmp_path / "run.ck2"
    a.save_checkpoint_v2(ck)
    b = trainer(cfg, hand_table)
    b.load_checkpoint_v2(ck)
    assert b.iterations_done == 3
    rows_equal(b.export_rows(), a.export_rows())
    b.train(2, 2048, verbose=False)  # iterations 4 and 5, linear-CFR weights included
    rows_equal(b.export_rows(), straight.export_rows())
    for t in (straight, a, b):
        t.close()


def test_train_checkpoints_carry_the_iteration(hand_table, tmp_path):
    """train() with a checkpoint interval writes v2 files for 64-bit keys, and
    the iteration count after it is the iterations run (not counted twice)."""
    cfg = L.preset(L.PRESET_HU_20BB)
    cfg.table_log2, cfg.key_bits = 20, 19
    a = trainer(cfg, hand_table)
    ck = tmp_path / "auto.ck2"
    a.train(4, 2048, verbose=False, ckpt_path=str(ck), ckpt_interval=2)
    assert a.stats().iterations_done == 4
    b = trainer(cfg, hand_table)
    b.load_checkpoint_v2(ck)
    assert b.iterations_done == 4
    rows_equal(b.export_rows(), a.export_rows())
    a.train(1, 2048, verbose=False)
    b.train(1, 2048, verbose=False)
    rows_equal(b.export_rows(), a.export_rows())
    a.close()
    b.close()


def test_refuses_other_games_and_bad_files(hand_table, tmp_path):
    cfg = L.preset(L.PRESET_HU_20BB)
    cfg.table_log2, cfg.key_bits = 20, 19
    a = trainer(cfg, hand_table)
    a.train(2, 2048, verbose=False)
    ck = tmp_path / "run.ck2"
    a.save_checkpoint_v2(ck)
    raw = ck.read_bytes()
    header = 8 + 4 + 4 + ctypes.sizeof(L.Config) + 8
    n = int(np.frombuffer(raw[header:header + 8], np.uint64)[0])
    assert n > 0 and len(raw) == header + 8 + 80 * n

    other = L.Config.from_buffer_copy(cfg)
    other.seed += 1
    c = trainer(other, hand_table)
    with pytest.raises(L.MccfrError) as e:
        c.load_checkpoint_v2(ck)
    assert e.value.status == ERR_INVALID_ARG

    d = trainer(cfg, hand_table)
    cut = tmp_path / "cut.ck2"
    cut.write_bytes(raw[: len(raw) - 40])
    with pytest.raises(L.MccfrError) as e:
        d.load_checkpoint_v2(cut)
    assert e.value.status == ERR_FORMAT

    bad = bytearray(raw)
    last = header + 8 + 80 * (n - 1)
    bad[last:last + 8] = np.array([(1 << 19) + 1], np.uint64).tobytes()  # past the 2^19-key space
    wild = tmp_path / "wild.ck2"
    wild.write_bytes(bytes(bad))
    with pytest.raises(L.MccfrError) as e:
        d.load_checkpoint_v2(wild)
    assert e.value.status == ERR_FORMAT
    d.load_checkpoint_v2(ck)  # the handle is still usable
    rows_equal(d.export_rows(), a.export_rows())
    for t in (a, c, d):
        t.close()


def test_reference_checkpoint_replaces_a_trained_table(hand_table, tmp_path):
    """Loading the reference-layout checkpoint into a handle that has trained
    on its own replaces every row, as the reference's load overwrites both
    arrays (cfr_gpu.cu:1526-1527): afterwards the handle holds exactly the
    saved rows, none of its own."""
    cfg = L.preset(L.PRESET_REF8)
    cfg.table_log2 = 26
    a = trainer(cfg, hand_table)
    a.train(2, 4096, verbose=False)
    ck = tmp_path / "a.ckpt"
    assert a.save_checkpoint(str(ck))
    b_cfg = L.Config.from_buffer_copy(cfg)
    b_cfg.seed = 7  # other deals: rows that A never touched
    b = trainer(b_cfg, hand_table)
    b.train(3, 4096, verbose=False)
    assert b.load_checkpoint(str(ck))
    ra, rb = a.export_rows(), b.export_rows()
    live = (np.abs(ra["regrets"]).sum(1) + np.abs(ra["strategy_sum"]).sum(1)) > 0
    assert np.array_equal(ra["keys"][live], rb["keys"])
    assert np.array_equal(ra["regrets"][live].view(np.uint32), rb["regrets"].view(np.uint32))
    assert np.array_equal(ra["strategy_sum"][live].view(np.uint32), rb["strategy_sum"].view(np.uint32))
    a.close()
    b.close()
