"""Showdown microbenchmark kernels against the oracle, bit for bit: the device's
seeded 7-card hands and their ranks, and the 6-seat shared-board winner masks of
training's own deals (checked against orc_showdown_masks)."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

import binding
from conftest import mccfr

L = mccfr.lib
pytestmark = pytest.mark.gpu


def trainer(cfg, table):
    t = mccfr.GPUCFRTrainer(config=cfg)
    t.set_hand_table(table)
    return t


def test_deal_eval7_equals_oracle(hand_table):
    import torch

    cfg = L.preset(L.PRESET_HU_20BB)
    cfg.seed, cfg.table_log2 = 3, 10
    tr = trainer(cfg, hand_table)
    lib = L.load()
    n = 1 << 18
    for stream in (0, 7):
        ranks = torch.empty(n, dtype=torch.int16, device="cuda")
        torch.cuda.synchronize()
        ms = ctypes.c_float()
        L.check(lib.mccfr_deal_eval7(tr.handle, stream, n, ctypes.c_void_p(ranks.data_ptr()), ctypes.byref(ms)))
        got = ranks.cpu().numpy().view(np.uint16)
        want = binding.deal_eval7(hand_table, 3, stream, n)
        assert np.array_equal(got, want), stream
        assert got.min() >= 1 and got.max() <= 7462 and ms.value > 0
    tr.close()


@pytest.mark.parametrize("iteration,player", [(1, 0), (2, 3)])
def test_showdown_masks_equal_oracle(hand_table, iteration, player):
    import torch

    cfg = L.preset(L.PRESET_6MAX_100BB)
    cfg.seed, cfg.table_log2 = 3, 12
    tr = trainer(cfg, hand_table)
    orc = binding.Oracle(cfg, hand_table)
    lib = L.load()
    n = 1 << 18
    masks = torch.empty(n, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    L.check(lib.mccfr_showdown_masks(tr.handle, iteration, player, n, ctypes.c_void_p(masks.data_ptr()), None))
    got = masks.cpu().numpy()
    want = orc.showdown_masks(iteration, player, n)
    assert np.array_equal(got, want)
    assert np.all((got > 0) & (got < 64))
    tr.close()
    orc.close()
