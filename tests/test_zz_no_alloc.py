"""mccfr_eval7_static: the evaluation entry point that allocates no device memory.

It exists for callers that cannot call cudaMalloc themselves (code running
inside a framework that owns every device allocation, or a process that must not
grow its device footprint).  Here the rank table is put on the device by torch's
allocator, standing in for such a framework, and the entry point is called
through the C ABI twice in a row; its ranks must equal those of mccfr_eval7, the
allocating entry point, exactly (integer ranks).  This file is collected last so
that a failure here cannot hide the other tests' results.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import mccfr

L = mccfr.lib
pytestmark = pytest.mark.gpu


def test_static_entry_point_matches_allocating_one(hand_table):
    import torch

    lib = L.load()
    dev_table = torch.from_numpy(hand_table).to("cuda:0")
    cfg = L.preset(L.PRESET_REF8)
    cfg.table_log2 = 12
    tr = mccfr.GPUCFRTrainer(config=cfg)
    tr.set_hand_table(hand_table)
    rng = np.random.default_rng(99)
    for call, n in enumerate((L.EVAL7_STATIC_MAX_HANDS, 12345)):
        cards = np.argsort(rng.random((n, 52)), axis=1)[:, :7].astype(np.uint8)
        want = tr.eval7(cards)
        got = np.full(n, 0xFFFF, dtype=np.uint16)
        torch.cuda.set_device(0)
        rc = lib.mccfr_eval7_static(L.c_void_p(dev_table.data_ptr()), L.ptr(cards), L.ptr(got), n)
        assert rc == L.OK, f"call {call}: status {rc}"
        assert np.array_equal(got, want), f"call {call} differs"
    # sizes beyond the static maximum are rejected, not truncated
    n = L.EVAL7_STATIC_MAX_HANDS + 1
    cards = np.zeros((n, 7), dtype=np.uint8)
    out = np.zeros(n, dtype=np.uint16)
    assert lib.mccfr_eval7_static(L.c_void_p(dev_table.data_ptr()), L.ptr(cards), L.ptr(out), n) == 1
    # a host copy of the table is refused before any kernel could read it
    cards = np.zeros((4, 7), dtype=np.uint8)
    cards[:] = np.arange(7)
    out = np.zeros(4, dtype=np.uint16)
    assert lib.mccfr_eval7_static(L.ptr(hand_table), L.ptr(cards), L.ptr(out), 4) == 1
    tr.close()
