"""ctypes bindings of libmccfr.so (declarations in include/mccfr.h).

The library is the product: loading fails loudly when it is missing, and no
Python path computes what a kernel computes.
"""
from __future__ import annotations

import ctypes
from ctypes import (POINTER, Structure, c_char_p, c_double, c_float, c_int, c_int32, c_int64,
                    c_longlong, c_size_t, c_uint8, c_uint32, c_uint64, c_void_p)
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "libmccfr.so"

HAND_TABLE_ENTRIES = 32487834
REF_TABLE_SIZE = 1 << 26

OK = 0
ERR = {
    1: "invalid argument", 2: "CUDA error", 3: "out of device memory", 4: "file I/O error",
    5: "bad file format", 6: "hand-rank table not loaded", 7: "info-set table full",
    8: "device-side error flag", 9: "accumulator range exceeded", 10: "output buffer too small",
    11: "no CUDA device", 12: "timeout",
}
ERR_CAPACITY = 10
ERR_NO_DEVICE = 11

ACT_FOLD, ACT_CHECK, ACT_CALL, ACT_CHECK_CALL, ACT_RAISE_MIN, ACT_RAISE_POT, ACT_ALL_IN = range(7)
SAMPLING_REFERENCE, SAMPLING_EXTERNAL = 0, 1
KEY_FNV26, KEY_ID64 = 0, 1
PREFLOP_CHEN64, PREFLOP_CLASS169 = 0, 1
POSTFLOP_REF_LINEAR, POSTFLOP_RANK_CDF = 0, 1
PRESET_REF8, PRESET_HU_20BB, PRESET_6MAX_100BB = 0, 1, 2
FORM_AUTO, FORM_LANES, FORM_LEVELS = 0, 1, 2
BATCH_PERSISTENT, BATCH_TABLE_GRAPHS = 0, 1


class Config(Structure):
    _fields_ = [
        ("num_players", c_int32), ("starting_stack", c_int32), ("small_blind", c_int32),
        ("big_blind", c_int32), ("use_cfr_plus", c_int32), ("use_linear_cfr", c_int32),
        ("sampling", c_int32), ("key_mode", c_int32), ("num_actions", c_int32),
        ("action_kind", c_int32 * 8), ("action_num", c_int32 * 8), ("action_den", c_int32 * 8),
        ("raise_cap", c_int32), ("max_depth", c_int32), ("preflop_mode", c_int32),
        ("preflop_buckets", c_int32), ("postflop_mode", c_int32), ("postflop_buckets", c_int32 * 3),
        ("table_log2", c_int32), ("device", c_int32), ("seed", c_uint64),
        ("key_bits", c_int32), ("traversal_form", c_int32), ("level_log2", c_int32),
        ("reserved", c_int32 * 5),
    ]

    def as_dict(self) -> dict:
        out = {}
        for name, _ in self._fields_:
            v = getattr(self, name)
            out[name] = list(v) if hasattr(v, "__len__") else v
        return out


class Stats(Structure):
    _fields_ = [
        ("iterations_done", c_int64), ("launches", c_int64), ("traversals", c_int64),
        ("node_visits", c_int64), ("traverser_updates", c_int64), ("terminals", c_int64),
        ("hand_evals", c_int64), ("rows_used", c_int64), ("table_capacity", c_int64),
        ("touched_last", c_int64), ("traverse_ms", c_double), ("apply_ms", c_double),
        ("last_traverse_ms", c_double), ("last_apply_ms", c_double), ("device_error", c_int32),
        ("wide_rows_last", c_int32), ("reserved", c_int32 * 6),
    ]


class BatchTuning(Structure):
    _fields_ = [("block", c_int32), ("grab", c_int32), ("smem_frames", c_int32), ("probe_width", c_int32),
                ("warp_sync", c_int32), ("form", c_int32), ("reserved", c_int32 * 2)]

    def as_dict(self) -> dict:
        return {"block": self.block, "grab": self.grab, "smem_frames": self.smem_frames,
                "probe_width": self.probe_width, "warp_sync": self.warp_sync, "form": self.form}


class BatchStats(Structure):
    _fields_ = [("iterations", c_int64), ("traversals", c_int64), ("node_visits", c_int64),
                ("traverse_ms", c_double), ("total_ms", c_double), ("reserved", c_int32 * 8)]


class Subgame(Structure):
    _fields_ = [("street", c_int32), ("pot", c_int32), ("board", c_uint8 * 5), ("pad", c_uint8 * 3),
                ("ranges", c_void_p)]


class BrOptions(Structure):
    _fields_ = [("threads", c_int32), ("flop_stride", c_int32), ("flags", c_int32), ("reserved", c_int32 * 5)]


BR_VERBOSE, BR_ISO_CHECK = 1, 2


class Exploit(Structure):
    _fields_ = [("br_value", c_double * 2), ("profile_value", c_double * 2), ("exploitability", c_double),
                ("mbb_per_game", c_double), ("seconds", c_double), ("iso_check", c_double),
                ("boards", c_longlong), ("rows", c_longlong), ("nodes", c_longlong), ("threads", c_int32),
                ("exact", c_int32), ("reserved", c_int32 * 4)]

    def as_dict(self) -> dict:
        return {"br_value": list(self.br_value), "profile_value": list(self.profile_value),
                "exploitability": self.exploitability, "mbb_per_game": self.mbb_per_game,
                "seconds": self.seconds, "iso_check": self.iso_check, "boards": self.boards, "rows": self.rows,
                "nodes": self.nodes, "threads": self.threads, "exact": bool(self.exact)}


class Trace(Structure):
    _fields_ = [
        ("hole", c_uint8 * 12), ("board", c_uint8 * 5), ("dealer", c_uint8), ("n_actions", c_uint8),
        ("n_traverser_nodes", c_uint8), ("hole_bucket", c_uint8 * 6), ("board_bucket", c_uint8 * 24),
        ("actions", c_uint8 * 40), ("payoff", c_float), ("reserved", c_uint32),
    ]


TRACE_DTYPE = np.dtype([
    ("hole", np.uint8, 12), ("board", np.uint8, 5), ("dealer", np.uint8), ("n_actions", np.uint8),
    ("n_traverser_nodes", np.uint8), ("hole_bucket", np.uint8, 6), ("board_bucket", np.uint8, (6, 4)),
    ("actions", np.uint8, 40), ("payoff", np.float32), ("reserved", np.uint32),
], align=True)
assert TRACE_DTYPE.itemsize == ctypes.sizeof(Trace), (TRACE_DTYPE.itemsize, ctypes.sizeof(Trace))

# Every function declared in include/mccfr.h: name -> (restype, argtypes)
SIGNATURES = {
    "mccfr_config_init": (c_int, [POINTER(Config), c_int]),
    "mccfr_config_validate": (c_int, [POINTER(Config), ctypes.c_char_p, c_size_t]),
    "mccfr_create": (c_int, [POINTER(Config), POINTER(c_void_p)]),
    "mccfr_destroy": (None, [c_void_p]),
    "mccfr_load_hand_table": (c_int, [c_void_p, c_char_p]),
    "mccfr_set_hand_table": (c_int, [c_void_p, c_void_p, c_size_t]),
    "mccfr_hand_table_generate": (c_int, [c_void_p, c_size_t]),
    "mccfr_hand_table_write": (c_int, [c_char_p]),
    "mccfr_hand_class_count": (c_int, []),
    "mccfr_train": (c_int, [c_void_p, c_longlong, c_int, c_int, c_char_p, c_longlong]),
    "mccfr_step": (c_int, [c_void_p, c_longlong, c_int, c_int, c_void_p]),
    "mccfr_get_strategy": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_size_t, POINTER(c_size_t)]),
    "mccfr_num_info_sets_active": (c_int, [c_void_p, POINTER(c_longlong)]),
    "mccfr_export_rows": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_size_t, POINTER(c_size_t)]),
    "mccfr_table_digest": (c_int, [c_void_p, c_void_p, c_void_p]),
    "mccfr_deal_eval7": (c_int, [c_void_p, c_uint32, c_size_t, c_void_p, POINTER(c_float)]),
    "mccfr_level_counts": (c_int, [c_void_p, c_void_p, c_void_p, c_int, POINTER(c_int), POINTER(c_uint32)]),
    "mccfr_showdown_masks": (c_int, [c_void_p, c_longlong, c_int, c_size_t, c_void_p, POINTER(c_float)]),
    "mccfr_export_tables": (c_int, [c_void_p, c_void_p, c_void_p, c_size_t]),
    "mccfr_import_tables": (c_int, [c_void_p, c_void_p, c_void_p, c_size_t]),
    "mccfr_save_checkpoint": (c_int, [c_void_p, c_char_p]),
    "mccfr_load_checkpoint": (c_int, [c_void_p, c_char_p]),
    "mccfr_save_checkpoint_v2": (c_int, [c_void_p, c_char_p]),
    "mccfr_load_checkpoint_v2": (c_int, [c_void_p, c_char_p]),
    "mccfr_save_strategy": (c_int, [c_void_p, c_char_p]),
    "mccfr_get_stats": (c_int, [c_void_p, POINTER(Stats)]),
    "mccfr_get_config": (c_int, [c_void_p, POINTER(Config)]),
    "mccfr_strerror": (c_char_p, [c_int]),
    "mccfr_last_error": (c_char_p, [c_void_p]),
    "mccfr_get_stream": (c_int, [c_void_p, POINTER(c_void_p)]),
    "mccfr_abi_sizes": (c_int, [c_void_p]),
    "mccfr_eval7": (c_int, [c_void_p, c_void_p, c_void_p, c_size_t]),
    "mccfr_eval7_device": (c_int, [c_void_p, c_void_p, c_void_p, c_size_t, POINTER(c_float)]),
    "mccfr_eval7_static": (c_int, [c_void_p, c_void_p, c_void_p, c_size_t]),
    "mccfr_batch_create": (c_int, [c_void_p, c_int, c_void_p, POINTER(c_void_p)]),
    "mccfr_batch_destroy": (None, [c_void_p]),
    "mccfr_batch_set_tuning": (c_int, [c_void_p, c_void_p]),
    "mccfr_batch_get_tuning": (c_int, [c_void_p, c_void_p]),
    "mccfr_batch_train": (c_int, [c_void_p, c_longlong, c_int]),
    "mccfr_batch_autotune": (c_int, [c_void_p, c_int, c_void_p]),
    "mccfr_batch_get_stats": (c_int, [c_void_p, c_void_p]),
    "mccfr_create_subgame": (c_int, [POINTER(Config), c_void_p, POINTER(c_void_p)]),
    "mccfr_share_hand_table": (c_int, [c_void_p, c_void_p]),
    "mccfr_batch_round": (c_int, [c_void_p, c_int, c_void_p, c_void_p]),
    "mccfr_get_progress": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    "mccfr_subgame_reset": (c_int, [c_void_p, c_void_p, c_void_p]),
    "mccfr_br_options_init": (None, [c_void_p]),
    "mccfr_best_response": (c_int, [c_void_p, c_void_p, c_void_p, c_size_t, c_void_p, c_void_p, c_size_t,
                                    c_void_p, c_void_p]),
    "mccfr_exploitability": (c_int, [c_void_p, c_void_p, c_void_p]),
    "mccfr_rank_cdf_lut": (c_int, [c_void_p, c_size_t, c_int, c_int, c_void_p]),
}
EVAL7_STATIC_MAX_HANDS = 1 << 18

_lib = None


def load() -> ctypes.CDLL:
    """Loads libmccfr.so (built by build.py); raises if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(f"{LIB_PATH} is missing: run build() first (no CPU fallback exists)")
    lib = ctypes.CDLL(str(LIB_PATH))
    for name, (res, args) in SIGNATURES.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


class MccfrError(RuntimeError):
    def __init__(self, status: int, message: str = ""):
        self.status = status
        super().__init__(f"{ERR.get(status, 'status %d' % status)}: {message}".rstrip(": "))


def check(status: int, handle=None) -> None:
    if status != OK:
        msg = ""
        if handle is not None:
            raw = load().mccfr_last_error(handle)
            msg = raw.decode() if raw else ""
        raise MccfrError(status, msg)


def preset(p: int) -> Config:
    cfg = Config()
    check(load().mccfr_config_init(ctypes.byref(cfg), p))
    return cfg


def validate(cfg: Config) -> str | None:
    """None for a valid config, else the first rule it breaks (no device needed)."""
    why = ctypes.create_string_buffer(256)
    rc = load().mccfr_config_validate(ctypes.byref(cfg), why, len(why))
    return None if rc == OK else why.value.decode()


def ptr(a: np.ndarray) -> c_void_p:
    return c_void_p(a.ctypes.data)


def generate_hand_table() -> np.ndarray:
    """The 32,487,834-entry rank table, built on the host by the library."""
    t = np.empty(HAND_TABLE_ENTRIES, dtype=np.int32)
    check(load().mccfr_hand_table_generate(ptr(t), t.size))
    return t


_TABLE_CACHE: np.ndarray | None = None


def hand_table() -> np.ndarray:
    global _TABLE_CACHE
    if _TABLE_CACHE is None:
        _TABLE_CACHE = generate_hand_table()
    return _TABLE_CACHE


def br_options(threads: int = 0, flop_stride: int = 1, verbose: bool = False, iso_check: bool = False) -> BrOptions:
    o = BrOptions()
    o.threads = int(threads)
    o.flop_stride = int(flop_stride)
    o.flags = (BR_VERBOSE if verbose else 0) | (BR_ISO_CHECK if iso_check else 0)
    return o


def subgame_struct(street: int, pot: int, board, ranges: np.ndarray) -> tuple[Subgame, np.ndarray]:
    """A Subgame struct and the float32 range array it points to (keep both alive)."""
    r = np.ascontiguousarray(ranges, dtype=np.float32)
    sg = Subgame()
    sg.street = int(street)
    sg.pot = int(pot)
    for i, c in enumerate(list(board)[:5]):
        sg.board[i] = int(c)
    sg.ranges = r.ctypes.data
    return sg, r


def best_response(config: Config, hand_table_: np.ndarray, keys: np.ndarray, strategy_sum: np.ndarray,
                  subgame: dict | None = None, **opts) -> dict:
    """Heads-up best response of rows (keys, strategy_sum [n][8]) on the host
    (mccfr_best_response); subgame = dict(street, pot, board, ranges) or None
    for the full game."""
    lib = load()
    t = np.ascontiguousarray(hand_table_, dtype=np.int32)
    k = np.ascontiguousarray(keys, dtype=np.uint64)
    s = np.ascontiguousarray(strategy_sum, dtype=np.float32).reshape(-1, 8)
    sgp = None
    if subgame is not None:
        sg, _keep = subgame_struct(subgame["street"], subgame["pot"], subgame["board"], subgame["ranges"])
        sgp = ctypes.byref(sg)
    out = Exploit()
    check(lib.mccfr_best_response(ctypes.byref(config), sgp, ptr(t), t.size, ptr(k), ptr(s), k.size,
                                  ctypes.byref(br_options(**opts)), ctypes.byref(out)))
    return out.as_dict()


def rank_cdf_lut(hand_table_: np.ndarray, ncards: int, buckets: int) -> np.ndarray:
    t = np.ascontiguousarray(hand_table_, dtype=np.int32)
    out = np.zeros(7463, dtype=np.uint8)
    check(load().mccfr_rank_cdf_lut(ptr(t), t.size, int(ncards), int(buckets), ptr(out)))
    return out
