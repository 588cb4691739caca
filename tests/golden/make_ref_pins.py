"""Generates tests/golden/ref_pins.npz from the reference's own CPU code.

Run in a container that has the reference sources (oracle/_ref/libref.so is
built from poker_cuda/src/hand_eval.cpp and abstraction.cpp by `make -C oracle
ref`).  The fixture records, on seeded random inputs:
  * evaluate_7cards (hand_eval.cpp:134-143) on the library-generated rank table,
  * evaluate_best with 3 and 4 community cards (hand_eval.cpp:149-173), whose
    5- and 6-card chains decode table states (the reference's own behaviour),
  * fast_postflop_bucket (abstraction.cpp:64-73),
  * preflop_bucket for every ordered hole pair (abstraction.cpp:55-59),
  * valid_actions_mask and action_to_chips (abstraction.cpp:167-234) on random
    betting states.
Usage: python tests/golden/make_ref_pins.py
"""
from __future__ import annotations

import ctypes
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT / "oracle"))
sys.path.insert(0, str(ROOT / "tests"))

import binding  # noqa: E402
from conftest import mccfr  # noqa: E402  (builds and registers the package)


def main() -> None:
    table = mccfr.hand_table()
    with tempfile.TemporaryDirectory() as d:
        path = Path(d) / "handranks.dat"
        table.tofile(path)
        ref = binding.ref()
        assert ref.ref_hand_eval_init(str(path).encode()) == 1
        rng = np.random.default_rng(20261203)
        n = 8000
        cards = np.stack([rng.permutation(52)[:7] for _ in range(n)]).astype(np.uint8)
        ev7 = np.array([ref.ref_evaluate_7cards(ctypes.c_void_p(cards[i].ctypes.data)) for i in range(n)],
                       dtype=np.uint16)
        best = np.zeros((n, 2), dtype=np.uint16)
        fast = np.zeros((n, 3), dtype=np.int16)
        for i in range(n):
            comm = np.ascontiguousarray(cards[i, 2:])
            cp = ctypes.c_void_p(comm.ctypes.data)
            best[i, 0] = ref.ref_evaluate_best(int(cards[i, 0]), int(cards[i, 1]), cp, 3)
            best[i, 1] = ref.ref_evaluate_best(int(cards[i, 0]), int(cards[i, 1]), cp, 4)
            for s, nc in enumerate((3, 4, 5)):
                fast[i, s] = ref.ref_fast_postflop_bucket(int(cards[i, 0]), int(cards[i, 1]), cp, nc)
        pre = np.zeros((52, 52), dtype=np.uint8)
        for a in range(52):
            for b in range(52):
                pre[a, b] = 0 if a == b else ref.ref_preflop_bucket(a, b)
        m = 16000
        bb = rng.choice([2, 10, 20, 100], size=m)
        stack = rng.integers(0, 3000, size=m)
        cb = rng.integers(0, 1500, size=m) * rng.integers(0, 2, size=m)
        to_call = np.minimum(cb, rng.integers(0, 3000, size=m))
        pot = rng.integers(-5, 6000, size=m)
        lfr = rng.integers(0, 800, size=m)
        states = np.stack([pot, stack, to_call, cb, lfr, bb], axis=1).astype(np.int32)
        masks = np.array([ref.ref_valid_actions_mask(*map(int, s)) for s in states], dtype=np.int32)
        chips = np.array([[ref.ref_action_to_chips(a, *map(int, s)) for a in range(8)] for s in states],
                         dtype=np.int32)
    np.savez_compressed(HERE / "ref_pins.npz", cards=cards, ev7=ev7, best=best, fast=fast, pre=pre,
                        states=states, masks=masks, chips=chips)
    print("wrote", HERE / "ref_pins.npz")


if __name__ == "__main__":
    main()
