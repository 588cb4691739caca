"""ctypes binding of the oracle (liboracle.so) and of the reference shim (_ref/libref.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg, as the checker.  The product never imports it.
"""
from __future__ import annotations

import ctypes
from ctypes import POINTER, c_char_p, c_float, c_int, c_int64, c_longlong, c_size_t, c_uint32, c_void_p
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_LIB = HERE / "liboracle.so"
REF_LIB = HERE / "_ref" / "libref.so"
REF_EVAL_LIB = HERE / "_ref" / "libref_eval.so"


def _p(a: np.ndarray) -> c_void_p:
    return c_void_p(a.ctypes.data)


_orc = None


def lib() -> ctypes.CDLL:
    global _orc
    if _orc is None:
        if not ORACLE_LIB.exists():
            raise RuntimeError(f"{ORACLE_LIB} missing: run `make -C oracle`")
        o = ctypes.CDLL(str(ORACLE_LIB))
        o.orc_create.restype = c_void_p
        o.orc_create.argtypes = [c_void_p, c_void_p]
        o.orc_destroy.argtypes = [c_void_p]
        o.orc_set_float_mode.argtypes = [c_void_p, c_int]
        o.orc_step.argtypes = [c_void_p, c_longlong, c_int, c_int, c_void_p, c_int]
        o.orc_step_wave.argtypes = [c_void_p, c_longlong, c_int, c_int, c_int]
        o.orc_wave_hist.argtypes = [c_void_p, c_void_p, c_int]
        o.orc_showdown_masks.argtypes = [c_void_p, c_longlong, c_int, c_int, c_void_p]
        o.orc_train.argtypes = [c_void_p, c_longlong, c_int, c_int]
        o.orc_counters.argtypes = [c_void_p, c_void_p]
        o.orc_export_rows.argtypes = [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_size_t, POINTER(c_size_t)]
        o.orc_table_digest.argtypes = [c_void_p, c_void_p, c_void_p]
        o.orc_config_init.argtypes = [c_void_p, c_int]
        o.orc_deal_eval7.argtypes = [c_void_p, ctypes.c_uint64, c_uint32, c_size_t, c_void_p]
        o.orc_hand_table_generate.argtypes = [c_void_p, c_size_t]
        o.orc_import_rows.argtypes = [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_size_t, c_longlong]
        o.orc_get_strategy.argtypes = [c_void_p, c_void_p, c_void_p, c_void_p, c_size_t, POINTER(c_size_t)]
        o.orc_philox.argtypes = [c_void_p, c_void_p, c_void_p]
        o.orc_uniform01.restype = c_float
        o.orc_uniform01.argtypes = [c_uint32]
        o.orc_eval7.argtypes = [c_void_p, c_void_p, c_void_p, c_size_t]
        o.orc_ref_board_bucket.argtypes = [c_void_p, c_int, c_int, c_void_p, c_int, c_int]
        o.orc_preflop_lut.argtypes = [c_int, c_int, c_void_p]
        o.orc_rank_cdf_lut.argtypes = [c_void_p, c_int, c_int, c_void_p]
        o.orc_rank_hist.argtypes = [c_void_p, c_int, c_void_p]
        o.orc_chain_rank.argtypes = [c_void_p, c_void_p, c_int]
        o.orc_valid_mask.argtypes = [c_void_p, c_int, c_int, c_int, c_int, c_int, c_int]
        o.orc_chips.argtypes = [c_void_p, c_int, c_int, c_int, c_int, c_int, c_int]
        o.orc_regret_frac_bits.argtypes = [c_void_p, c_longlong]
        o.orc_create_subgame.restype = c_void_p
        o.orc_create_subgame.argtypes = [c_void_p, c_void_p, c_int, c_int, c_void_p, c_void_p]
        o.orc_range_cdf.argtypes = [c_void_p, c_void_p, c_int, c_void_p]
        o.brute_rank.argtypes = [c_void_p, c_int]
        o.brute_rank_batch.argtypes = [c_void_p, c_int, c_void_p, c_size_t, c_int]
        _orc = o
    return _orc


class Oracle:
    """CPU restatement of one trainer (same config struct as the product)."""

    def __init__(self, config, hand_table: np.ndarray, subgame: dict | None = None):
        self._t = np.ascontiguousarray(hand_table, dtype=np.int32)  # kept alive (borrowed by C)
        self._cfg = config
        if subgame is None:
            self._h = lib().orc_create(ctypes.byref(config), _p(self._t))
            return
        board = np.zeros(5, dtype=np.uint8)
        nb = 4 if subgame["street"] == 2 else 5
        board[:nb] = subgame["board"][:nb]
        ranges = np.ascontiguousarray(subgame["ranges"], dtype=np.float32).reshape(config.num_players, 1326)
        cdf = np.zeros((config.num_players, 1326), dtype=np.uint32)
        for p in range(config.num_players):
            assert lib().orc_range_cdf(_p(ranges[p]), _p(board), nb, _p(cdf[p])) == 1
        self._cdf = cdf
        self._h = lib().orc_create_subgame(ctypes.byref(config), _p(self._t), subgame["street"], subgame["pot"],
                                           _p(board), _p(cdf))

    def close(self):
        if self._h:
            lib().orc_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_float_mode(self, on: bool):
        lib().orc_set_float_mode(self._h, 1 if on else 0)

    def step(self, iteration: int, player: int, batch: int, trace: bool = False, threads: int = 8,
             trace_dtype=None):
        buf = np.zeros(batch, dtype=trace_dtype) if trace else None
        lib().orc_step(self._h, iteration, player, batch, _p(buf) if trace else None, threads)
        return buf

    def step_wave(self, iteration: int, player: int, batch: int, threads: int = 8) -> int:
        """The same player-update, expanded level by level (orc_step_wave);
        returns the status (integer-sum mode only)."""
        return lib().orc_step_wave(self._h, iteration, player, batch, threads)

    def showdown_masks(self, iteration: int, player: int, n: int) -> np.ndarray:
        """Winner masks (bit q: seat q holds the best rank) of the deals of
        traversals 0..n-1 of update (iteration, player)."""
        out = np.zeros(n, np.uint8)
        assert lib().orc_showdown_masks(self._h, iteration, player, n, _p(out)) == 0
        return out

    def wave_hist(self) -> np.ndarray:
        """Nodes per tree depth in the last level-synchronous update."""
        out = np.zeros(512, np.int64)
        n = lib().orc_wave_hist(self._h, _p(out), out.size)
        return out[: min(n, out.size)]

    def train(self, iters: int, batch: int, threads: int = 8):
        lib().orc_train(self._h, iters, batch, threads)

    def counters(self) -> dict:
        c = np.zeros(6, dtype=np.int64)
        lib().orc_counters(self._h, _p(c))
        return dict(zip(["traversals", "visits", "updates", "evals", "terminals", "rows"], c.tolist()))

    def export_rows(self) -> dict:
        n = c_size_t()
        lib().orc_export_rows(self._h, None, None, None, None, 0, ctypes.byref(n))
        m = n.value
        keys = np.empty(m, np.uint64)
        reg = np.empty((m, 8), np.float32)
        ssum = np.empty((m, 8), np.float32)
        vis = np.empty(m, np.uint64)
        lib().orc_export_rows(self._h, _p(keys), _p(reg), _p(ssum), _p(vis), m, ctypes.byref(n))
        return {"keys": keys, "regrets": reg, "strategy_sum": ssum, "visits": vis}

    def digest(self) -> tuple[int, int]:
        """(checksum, rows) of the table, the figures mccfr_table_digest gives
        for a device table with the same rows."""
        out = np.zeros(2, np.uint64)
        assert lib().orc_table_digest(self._h, _p(out[:1]), _p(out[1:])) == 0
        return int(out[0]), int(out[1])

    def import_rows(self, rows: dict, iterations_done: int = 0) -> None:
        """Replaces the table with `rows` (the dict export_rows returns, e.g. a
        device trainer's export) and sets the completed-iteration count."""
        keys = np.ascontiguousarray(rows["keys"], dtype=np.uint64)
        reg = np.ascontiguousarray(rows["regrets"], dtype=np.float32).reshape(-1, 8)
        ssum = np.ascontiguousarray(rows["strategy_sum"], dtype=np.float32).reshape(-1, 8)
        vis = np.ascontiguousarray(rows["visits"], dtype=np.uint64)
        n = keys.size
        assert reg.shape[0] == ssum.shape[0] == vis.size == n
        rc = lib().orc_import_rows(self._h, _p(keys), _p(reg), _p(ssum), _p(vis), n, iterations_done)
        if rc:
            raise ValueError(f"orc_import_rows: status {rc}")

    def strategy_arrays(self):
        n = c_size_t()
        lib().orc_get_strategy(self._h, None, None, None, 0, ctypes.byref(n))
        m = n.value
        keys = np.empty(m, np.uint32)
        probs = np.empty((m, 8), np.float32)
        lib().orc_get_strategy(self._h, _p(keys), None, _p(probs), m, ctypes.byref(n))
        return keys[: n.value], probs[: n.value]


def config_init(cfg, preset: int):
    """Fills a config struct (the ctypes mirror of mccfr_config) with one of the
    three presets, without the device library."""
    rc = lib().orc_config_init(ctypes.byref(cfg), int(preset))
    if rc:
        raise ValueError(f"orc_config_init: status {rc}")
    return cfg


HAND_TABLE_ENTRIES = 32487834


def hand_table() -> np.ndarray:
    """The 32,487,834-entry rank table, built on the host by the oracle library."""
    t = np.empty(HAND_TABLE_ENTRIES, dtype=np.int32)
    rc = lib().orc_hand_table_generate(_p(t), t.size)
    if rc:
        raise RuntimeError(f"orc_hand_table_generate: status {rc}")
    return t


def philox(ctr, key) -> np.ndarray:
    c = np.asarray(ctr, dtype=np.uint32)
    k = np.asarray(key, dtype=np.uint32)
    out = np.zeros(4, dtype=np.uint32)
    lib().orc_philox(_p(c), _p(k), _p(out))
    return out


def eval7(table: np.ndarray, cards: np.ndarray) -> np.ndarray:
    c = np.ascontiguousarray(cards, dtype=np.uint8).reshape(-1, 7)
    out = np.empty(c.shape[0], dtype=np.uint16)
    lib().orc_eval7(_p(table), _p(c), _p(out), c.shape[0])
    return out


def deal_eval7(table: np.ndarray, seed: int, stream: int, n: int) -> np.ndarray:
    """Ranks of the showdown microbenchmark's hands 0..n-1 (orc_deal_eval7)."""
    out = np.empty(n, dtype=np.uint16)
    assert lib().orc_deal_eval7(_p(table), int(seed), int(stream), n, _p(out)) == 0
    return out


def brute_ranks(cards: np.ndarray, n: int, threads: int = 8) -> np.ndarray:
    c = np.ascontiguousarray(cards, dtype=np.uint8).reshape(-1, n)
    out = np.empty(c.shape[0], dtype=np.uint16)
    lib().brute_rank_batch(_p(c), n, _p(out), c.shape[0], threads)
    return out


def rank_hist(table: np.ndarray, ncards: int) -> np.ndarray:
    out = np.zeros(7463, dtype=np.uint64)
    lib().orc_rank_hist(_p(table), ncards, _p(out))
    return out


def preflop_lut(mode: int, buckets: int) -> np.ndarray:
    out = np.zeros(52 * 52, dtype=np.uint8)
    lib().orc_preflop_lut(mode, buckets, _p(out))
    return out


def chain_rank(table: np.ndarray, cards) -> int:
    c = np.ascontiguousarray(cards, dtype=np.uint8)
    return lib().orc_chain_rank(_p(table), _p(c), c.size)


def valid_mask(cfg, pot, stack, to_call, cb, lfr, raises=0) -> int:
    return lib().orc_valid_mask(ctypes.byref(cfg), pot, stack, to_call, cb, lfr, raises)


def chips(cfg, a, pot, stack, to_call, cb, lfr) -> int:
    return lib().orc_chips(ctypes.byref(cfg), a, pot, stack, to_call, cb, lfr)


# ---- the reference's own CPU functions (compiled from its sources) -----------
_ref = None


def ref_available() -> bool:
    return REF_LIB.exists()


def ref() -> ctypes.CDLL:
    global _ref
    if _ref is None:
        r = ctypes.CDLL(str(REF_LIB))
        r.ref_hand_eval_init.argtypes = [c_char_p]
        r.ref_evaluate_7cards.argtypes = [c_void_p]
        r.ref_evaluate_best.argtypes = [c_int, c_int, c_void_p, c_int]
        r.ref_preflop_bucket.argtypes = [c_int, c_int]
        r.ref_fast_postflop_bucket.argtypes = [c_int, c_int, c_void_p, c_int]
        r.ref_valid_actions_mask.argtypes = [c_int] * 6
        r.ref_action_to_chips.argtypes = [c_int] * 7
        r.ref_abstraction_init()
        _ref = r
    return _ref


_ref_eval = None

# OpponentType of the reference's eval.h, in order.
OPPONENTS = ("calling_station", "nit", "maniac", "balanced", "random")


def ref_eval_available() -> bool:
    return REF_EVAL_LIB.exists()


def ref_eval() -> ctypes.CDLL:
    """The reference's strategy loader and scripted-opponent evaluator
    (strategy.cpp, eval.cpp), compiled unchanged by oracle/Makefile."""
    global _ref_eval
    if _ref_eval is None:
        r = ctypes.CDLL(str(REF_EVAL_LIB))
        r.refeval_init.argtypes = [c_char_p]
        r.refeval_load.argtypes = [c_char_p]
        r.refeval_load.restype = c_longlong
        r.refeval_entry.argtypes = [c_uint32, c_void_p]
        r.refeval_play.argtypes = [c_int, c_int, c_longlong, c_int, c_int, c_int, ctypes.c_uint,
                                   POINTER(ctypes.c_double), POINTER(ctypes.c_double), POINTER(c_longlong)]
        _ref_eval = r
    return _ref_eval


def ref_play(opponent: str, n_hands: int, n_players: int = 2, stack: int = 1000, sb: int = 10, bb: int = 20,
             seed: int = 42) -> dict:
    """evaluate_strategy_np on the strategy loaded by ref_eval().refeval_load."""
    b100, net, hands = ctypes.c_double(), ctypes.c_double(), c_longlong()
    ref_eval().refeval_play(n_players, OPPONENTS.index(opponent), n_hands, stack, sb, bb, seed,
                            ctypes.byref(b100), ctypes.byref(net), ctypes.byref(hands))
    return {"bb_per_100": b100.value, "net_bb": net.value, "hands": hands.value}


def write_strategy_v2(path, keys32: np.ndarray, probs: np.ndarray) -> None:
    """The v2 strategy dump mccfr_save_strategy writes (include/mccfr.h):
    [u64 magic][u32 2^26][u32 8][u32 n] then n x {u32 key, f32[8]}, keys ascending."""
    order = np.argsort(keys32, kind="stable")
    rec = np.zeros(len(keys32), dtype=np.dtype([("k", np.uint32), ("p", np.float32, 8)]))
    rec["k"] = keys32[order]
    rec["p"] = probs[order]
    with open(path, "wb") as f:
        f.write(np.array([0x53545241540100], np.uint64).tobytes())
        f.write(np.array([1 << 26, 8, len(rec)], np.uint32).tobytes())
        f.write(rec.tobytes())
