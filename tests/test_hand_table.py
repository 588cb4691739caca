"""The generated 7-card rank table against brute force, published counts and
the reference's own evaluator (CPU)."""
from __future__ import annotations

import itertools

import numpy as np
import pytest

import binding
from conftest import mccfr

L = mccfr.lib

# Published best-hand category counts over all C(52,7) = 133,784,560 hands and
# all C(52,5) = 2,598,960 hands (high card .. straight flush incl. royal).
CAT7 = [23294460, 58627800, 31433400, 6461620, 6180020, 4047644, 3473184, 224848, 41584]
CAT5 = [1302540, 1098240, 123552, 54912, 10200, 5108, 3744, 624, 40]
CAT_BOUNDS = [1, 1278, 4138, 4996, 5854, 5864, 7141, 7297, 7453, 7463]


def rm(c: int) -> int:
    return (c % 13) * 4 + c // 13 + 1


def chain(T, cards):
    p = int(T[53 + rm(cards[0])])
    for c in cards[1:]:
        p = int(T[p + rm(c)])
    return p


def decode(v: int) -> int:
    v &= 0xFFFF
    cat, o = v >> 12, v & 0xFFF
    base = [0, 0, 1277, 4137, 4995, 5853, 5863, 7140, 7296, 7452]
    return 0 if (o == 0 or cat < 1 or cat > 9) else base[cat] + o


def categories(hist: np.ndarray) -> list[int]:
    return [int(hist[CAT_BOUNDS[i]:CAT_BOUNDS[i + 1]].sum()) for i in range(9)]


def test_size_kat_and_classes(hand_table):
    T = hand_table
    assert T.size == L.HAND_TABLE_ENTRIES == 32487834
    # As Ks Qs Js Ts 2c 3d -> 7462 (hand_eval.cpp:70-75, cfr_gpu.cu:279-288)
    assert decode(chain(T, [51, 50, 49, 48, 47, 0, 14])) == 7462
    assert L.load().mccfr_hand_class_count() == 7462
    assert binding.lib().brute_class_count() == 7462
    # 612,977 canonical partial hands fill the table exactly: the last state's row
    # is the final 53 entries and holds live transitions.
    assert np.count_nonzero(T[-52:]) > 0
    assert T[:53].max() == 0


def test_generation_is_deterministic(hand_table):
    again = L.generate_hand_table()
    assert np.array_equal(again, hand_table)


def test_exhaustive_category_counts(hand_table):
    h7 = binding.rank_hist(hand_table, 7)
    assert int(h7.sum()) == 133784560 and h7[0] == 0
    assert categories(h7) == CAT7
    h5 = binding.rank_hist(hand_table, 5)
    assert int(h5.sum()) == 2598960
    assert categories(h5) == CAT5
    # every one of the 7462 classes occurs among 5-card hands
    assert np.count_nonzero(h5[1:]) == 7462


def test_rank7_digests(hand_table):
    """The oracle's per-group digests of the exhaustive 7-card sweep (the GPU
    sweep's checker): their sums agree with the exhaustive histogram, and two
    groups agree with per-hand ranks in lexicographic order."""
    s = np.zeros(52 * 52, np.uint64)
    w = np.zeros(52 * 52, np.uint64)
    binding.lib().orc_rank7_digests(binding._p(hand_table), binding._p(s), binding._p(w))
    h7 = binding.rank_hist(hand_table, 7)
    assert int(s.sum()) == int((h7 * np.arange(7463, dtype=np.uint64)).sum())
    assert np.count_nonzero(s) == sum(b for b in range(1, 47))  # groups with 5 cards above b
    for a, b in ((0, 1), (30, 44)):
        tails = np.array(list(itertools.combinations(range(b + 1, 52), 5)), np.uint8)
        cards = np.concatenate([np.full((len(tails), 2), (a, b), np.uint8), tails], axis=1)
        r = binding.eval7(hand_table, cards).astype(np.uint64)
        assert int(r.sum()) == int(s[a * 52 + b])
        assert int((r * np.arange(1, len(r) + 1, dtype=np.uint64)).sum()) == int(w[a * 52 + b])


def test_against_brute_force(hand_table):
    rng = np.random.default_rng(7)
    cards = np.stack([rng.permutation(52)[:7] for _ in range(200000)]).astype(np.uint8)
    assert np.array_equal(binding.eval7(hand_table, cards), binding.brute_ranks(cards, 7))
    # 5- and 6-card ranks live at the state's card-0 entry
    for n in (5, 6):
        sub = np.ascontiguousarray(cards[:20000, :n])
        table_r = np.array([binding.chain_rank(hand_table, c) for c in sub], dtype=np.uint16)
        assert np.array_equal(table_r, binding.brute_ranks(sub, n))


def test_state_depends_only_on_card_set(hand_table):
    """The product walks the board first and shares it between players; the
    reference walks hole cards first (cfr_gpu.cu:114-150).  Every prefix state
    must be a function of the card set."""
    T = hand_table
    rng = np.random.default_rng(11)
    for _ in range(3000):
        c = [int(x) for x in rng.permutation(52)[:7]]
        for n in (5, 6, 7):
            base = chain(T, c[:n])
            for perm in itertools.islice(itertools.permutations(c[:n]), 0, 720, 97):
                assert chain(T, list(perm)) == base


def test_against_reference_pins(hand_table):
    """Fixtures produced by the reference's own hand_eval.cpp on this table."""
    pins = np.load(__import__("pathlib").Path(__file__).parent / "golden" / "ref_pins.npz")
    cards = pins["cards"]
    assert np.array_equal(binding.eval7(hand_table, cards), pins["ev7"])
    # evaluate_best with 3/4 community cards decodes the 5th/6th chain value
    # (a state, not a rank): the oracle restates that exactly.
    for i in range(cards.shape[0]):
        c = [int(x) for x in cards[i]]
        assert decode(chain(hand_table, c[:5])) == pins["best"][i, 0]
        assert decode(chain(hand_table, c[:6])) == pins["best"][i, 1]


@pytest.mark.skipif(not binding.ref_available(), reason="reference sources not built here")
def test_against_reference_live(hand_table, hand_table_file):
    ref = binding.ref()
    assert ref.ref_hand_eval_init(str(hand_table_file).encode()) == 1
    rng = np.random.default_rng(5)
    cards = np.stack([rng.permutation(52)[:7] for _ in range(5000)]).astype(np.uint8)
    got = np.array([ref.ref_evaluate_7cards(L.ptr(np.ascontiguousarray(c))) for c in cards])
    assert np.array_equal(got, binding.eval7(hand_table, cards))


def test_table_file_roundtrip(hand_table, tmp_path):
    p = tmp_path / "hr.dat"
    assert L.load().mccfr_hand_table_write(str(p).encode()) == 0
    assert p.stat().st_size == 129951336
    assert np.array_equal(np.fromfile(p, dtype=np.int32), hand_table)
