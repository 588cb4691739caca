"""Host mirror of the reference's trainer class over the C ABI.

`GPUCFRTrainer` keeps the constructor, method names, argument meaning and
return conventions of poker_cuda/src/cfr_gpu.cuh:48-132:
  * load_hand_table / save_checkpoint / load_checkpoint return bool, as there;
  * train(total_iterations, batch_size=65536, verbose=True, ckpt_path="",
    ckpt_interval=10000) as cfr_gpu.cu:1244;
  * get_strategy() returns {u32 key: float32[8]} like HostStrategyTable
    (cfr_gpu.cuh:30-33), rows with a zero sum skipped (cfr_gpu.cu:1399-1411);
  * num_info_sets_active(), export_tables(), import_tables().
Where the reference calls exit(1) on a CUDA error (cfr_gpu.cu:61-69) this class
raises MccfrError.  Extra keyword arguments select the seed, update rule and
abstraction preset that the reference hard-wires.
"""
from __future__ import annotations

import ctypes
import json
import time
from ctypes import byref, c_longlong, c_size_t, c_void_p

import numpy as np

from . import lib as L


class GPUCFRTrainer:
    def __init__(self, num_players: int = 2, starting_stack: int = 1000, small_blind: int = 10,
                 big_blind: int = 20, use_cfr_plus: bool = True, use_linear_cfr: bool = True, *,
                 preset: int = L.PRESET_REF8, config: L.Config | None = None, seed: int | None = None,
                 sampling: int | None = None, table_log2: int | None = None, device: int = 0):
        self._lib = L.load()
        if config is None:
            config = L.preset(preset)
            if preset == L.PRESET_REF8:
                config.num_players = num_players
                config.starting_stack = starting_stack
                config.small_blind = small_blind
                config.big_blind = big_blind
            config.use_cfr_plus = int(bool(use_cfr_plus))
            config.use_linear_cfr = int(bool(use_linear_cfr))
        if seed is not None:
            config.seed = int(seed)
        if sampling is not None:
            config.sampling = int(sampling)
        if table_log2 is not None:
            config.table_log2 = int(table_log2)
        config.device = int(device)
        self.config = config
        h = c_void_p()
        L.check(self._lib.mccfr_create(byref(config), byref(h)))
        self._h = h
        self.iterations_done = 0

    @classmethod
    def subgame(cls, config: L.Config, street: int, pot: int, board, ranges: np.ndarray) -> "GPUCFRTrainer":
        """A turn (street 2, 4 board cards) or river (street 3, 5 cards) subgame with
        one 1326-combo range per player (mccfr_create_subgame)."""
        self = cls.__new__(cls)
        self._lib = L.load()
        self.config = config
        sg, _keep = L.subgame_struct(street, pot, board,
                                     np.asarray(ranges, dtype=np.float32).reshape(config.num_players, 1326))
        h = c_void_p()
        L.check(self._lib.mccfr_create_subgame(byref(config), byref(sg), byref(h)))
        self._h = h
        self.iterations_done = 0
        return self

    def reset_subgame(self, config: L.Config, street: int, pot: int, board, ranges: np.ndarray) -> None:
        """Re-targets this subgame trainer to a new subgame with the same table
        capacity (mccfr_subgame_reset): as if freshly created, allocations kept."""
        sg, _keep = L.subgame_struct(street, pot, board,
                                     np.asarray(ranges, dtype=np.float32).reshape(config.num_players, 1326))
        L.check(self._lib.mccfr_subgame_reset(self._h, byref(config), byref(sg)), self._h)
        self.config = config
        self.iterations_done = 0

    def share_hand_table(self, src: "GPUCFRTrainer") -> None:
        L.check(self._lib.mccfr_share_hand_table(self._h, src.handle), self._h)

    def progress(self) -> tuple[int, int, int]:
        it, pl, done = ctypes.c_longlong(), ctypes.c_int(), ctypes.c_longlong()
        L.check(self._lib.mccfr_get_progress(self._h, byref(it), byref(pl), byref(done)), self._h)
        return it.value, pl.value, done.value

    # -- lifetime ------------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.mccfr_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self) -> c_void_p:
        return self._h

    # -- reference API -------------------------------------------------------
    def load_hand_table(self, path: str = "data/handranks.dat") -> bool:
        return self._lib.mccfr_load_hand_table(self._h, str(path).encode()) == L.OK

    def set_hand_table(self, table: np.ndarray) -> None:
        t = np.ascontiguousarray(table, dtype=np.int32)
        L.check(self._lib.mccfr_set_hand_table(self._h, L.ptr(t), t.size), self._h)

    def train(self, total_iterations: int, batch_size: int = 65536, verbose: bool = True,
              ckpt_path: str = "", ckpt_interval: int = 10000, timed: bool = False,
              metrics: str | None = None) -> None:
        """As the reference's train.  metrics: a JSON-lines file that gets one
        line for this call (metrics_line), with the kernels timed on the device."""
        timed = timed or metrics is not None
        s0 = self.stats() if metrics else None
        t0 = time.perf_counter()
        flags = (1 if verbose else 0) | (2 if timed else 0)
        L.check(self._lib.mccfr_train(self._h, int(total_iterations), int(batch_size), flags,
                                      ckpt_path.encode(), int(ckpt_interval)), self._h)
        self.iterations_done += int(total_iterations)
        if metrics:
            line = metrics_line(s0, self.stats(), time.perf_counter() - t0, int(total_iterations), int(batch_size))
            with open(metrics, "a") as f:
                f.write(json.dumps(line) + "\n")

    def get_strategy(self) -> dict[int, np.ndarray]:
        keys, probs = self.strategy_arrays()
        return {int(k): probs[i] for i, k in enumerate(keys)}

    def save_checkpoint(self, path: str) -> bool:
        return self._lib.mccfr_save_checkpoint(self._h, str(path).encode()) == L.OK

    def load_checkpoint(self, path: str) -> bool:
        return self._lib.mccfr_load_checkpoint(self._h, str(path).encode()) == L.OK

    def save_checkpoint_v2(self, path: str) -> None:
        """Config, iteration count and every occupied row (mccfr_save_checkpoint_v2)."""
        L.check(self._lib.mccfr_save_checkpoint_v2(self._h, str(path).encode()), self._h)

    def load_checkpoint_v2(self, path: str) -> None:
        """Replaces the table and the iteration count; training continues exactly
        where the saved trainer stopped (mccfr_load_checkpoint_v2)."""
        L.check(self._lib.mccfr_load_checkpoint_v2(self._h, str(path).encode()), self._h)
        self.iterations_done = int(self.stats().iterations_done)

    def num_info_sets_active(self) -> int:
        n = c_longlong()
        L.check(self._lib.mccfr_num_info_sets_active(self._h, byref(n)), self._h)
        return int(n.value)

    def export_tables(self) -> tuple[np.ndarray, np.ndarray]:
        n = 8 * L.REF_TABLE_SIZE
        r = np.empty(n, dtype=np.float32)
        s = np.empty(n, dtype=np.float32)
        L.check(self._lib.mccfr_export_tables(self._h, L.ptr(r), L.ptr(s), n), self._h)
        return r, s

    def import_tables(self, regrets: np.ndarray, strategy_sum: np.ndarray) -> None:
        r = np.ascontiguousarray(regrets, dtype=np.float32)
        s = np.ascontiguousarray(strategy_sum, dtype=np.float32)
        L.check(self._lib.mccfr_import_tables(self._h, L.ptr(r), L.ptr(s), r.size), self._h)

    # -- extensions ----------------------------------------------------------
    def step(self, iteration: int, player: int, batch: int, trace: bool = False):
        """One player-update; returns per-traversal trace records when asked."""
        buf = np.zeros(batch, dtype=L.TRACE_DTYPE) if trace else None
        L.check(self._lib.mccfr_step(self._h, int(iteration), int(player), int(batch),
                                     L.ptr(buf) if trace else None), self._h)
        return buf

    def strategy_arrays(self) -> tuple[np.ndarray, np.ndarray]:
        n = c_size_t()
        rc = self._lib.mccfr_get_strategy(self._h, None, None, None, 0, byref(n))
        if rc not in (L.OK, L.ERR_CAPACITY):
            L.check(rc, self._h)
        cap = n.value
        keys = np.empty(cap, dtype=np.uint32)
        probs = np.empty((cap, 8), dtype=np.float32)
        L.check(self._lib.mccfr_get_strategy(self._h, L.ptr(keys), None, L.ptr(probs), cap, byref(n)), self._h)
        return keys[: n.value], probs[: n.value]

    def rows_used(self) -> int:
        """Occupied rows of the info-set table, counted on the device (the
        size query of mccfr_export_rows: capacity 0, no copy)."""
        n = c_size_t()
        rc = self._lib.mccfr_export_rows(self._h, None, None, None, None, 0, byref(n))
        if rc not in (L.OK, L.ERR_CAPACITY):
            L.check(rc, self._h)
        return int(n.value)

    def export_rows(self) -> dict[str, np.ndarray]:
        n = c_size_t()
        rc = self._lib.mccfr_export_rows(self._h, None, None, None, None, 0, byref(n))
        if rc not in (L.OK, L.ERR_CAPACITY):
            L.check(rc, self._h)
        cap = n.value
        keys = np.empty(cap, dtype=np.uint64)
        reg = np.empty((cap, 8), dtype=np.float32)
        ssum = np.empty((cap, 8), dtype=np.float32)
        vis = np.empty(cap, dtype=np.uint64)
        L.check(self._lib.mccfr_export_rows(self._h, L.ptr(keys), L.ptr(reg), L.ptr(ssum), L.ptr(vis), cap,
                                            byref(n)), self._h)
        m = n.value
        return {"keys": keys[:m], "regrets": reg[:m], "strategy_sum": ssum[:m], "visits": vis[:m]}

    def level_counts(self) -> dict:
        """Per-level seeds and updating-player nodes of the last external-sampling
        update in the level-synchronous form (mccfr_level_counts)."""
        seeds = np.zeros(64, np.uint32)
        nodes = np.zeros(64, np.uint32)
        n, deferred = ctypes.c_int(), ctypes.c_uint32()
        L.check(self._lib.mccfr_level_counts(self._h, L.ptr(seeds), L.ptr(nodes), 64, byref(n), byref(deferred)),
                self._h)
        k = n.value
        return {"seeds": seeds[:k].tolist(), "nodes": nodes[:k].tolist(), "deferred": int(deferred.value)}

    def digest(self) -> tuple[int, int]:
        """(checksum, occupied rows) of the table, computed on the device
        (mccfr_table_digest): equal for tables with the same rows."""
        d, n = ctypes.c_uint64(), ctypes.c_uint64()
        L.check(self._lib.mccfr_table_digest(self._h, byref(d), byref(n)), self._h)
        return int(d.value), int(n.value)

    def save_strategy(self, path: str) -> bool:
        return self._lib.mccfr_save_strategy(self._h, str(path).encode()) == L.OK

    def stats(self) -> L.Stats:
        s = L.Stats()
        L.check(self._lib.mccfr_get_stats(self._h, byref(s)), self._h)
        return s

    def stream_ptr(self) -> int:
        p = c_void_p()
        L.check(self._lib.mccfr_get_stream(self._h, byref(p)), self._h)
        return int(p.value or 0)

    def exploitability(self, threads: int = 0, flop_stride: int = 1, verbose: bool = False,
                       iso_check: bool = False) -> dict:
        """Heads-up best response to the current average strategy, FP64 on host
        threads (mccfr_exploitability)."""
        out = L.Exploit()
        opts = L.br_options(threads, flop_stride, verbose, iso_check)
        L.check(self._lib.mccfr_exploitability(self._h, byref(opts), byref(out)), self._h)
        return out.as_dict()

    def eval7(self, cards: np.ndarray) -> np.ndarray:
        c = np.ascontiguousarray(cards, dtype=np.uint8).reshape(-1, 7)
        out = np.empty(c.shape[0], dtype=np.uint16)
        L.check(self._lib.mccfr_eval7(self._h, L.ptr(c), L.ptr(out), c.shape[0]), self._h)
        return out


class Batch:
    """Several trainers (tables) trained together, by one persistent kernel per
    phase or as concurrent branches of one graph (set_tuning(form=...)); each
    table's result equals training it alone (mccfr_batch_*)."""

    def __init__(self, trainers: list, traversals: list[int]):
        self._lib = L.load()
        self.trainers = list(trainers)  # keep the handles alive
        arr = (ctypes.c_void_p * len(trainers))(*[t.handle.value for t in trainers])
        cnt = (ctypes.c_int * len(traversals))(*[int(x) for x in traversals])
        b = c_void_p()
        rc = self._lib.mccfr_batch_create(arr, len(trainers), cnt, byref(b))
        L.check(rc)
        self._b = b

    def close(self) -> None:
        if getattr(self, "_b", None):
            self._lib.mccfr_batch_destroy(self._b)
            self._b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def train(self, iters: int, timed: bool = False) -> None:
        L.check(self._lib.mccfr_batch_train(self._b, int(iters), 2 if timed else 0))
        for t in self.trainers:
            t.iterations_done += int(iters)

    def autotune(self, max_candidates: int = 0) -> dict:
        best = L.BatchTuning()
        L.check(self._lib.mccfr_batch_autotune(self._b, int(max_candidates), byref(best)))
        n = 2 * len(self.candidates(max_candidates))  # forward and backward pass
        for t in self.trainers:
            t.iterations_done += n
        return best.as_dict()

    @staticmethod
    def candidates(max_candidates: int = 0) -> list:
        c = [dict(block=b, grab=g, smem_frames=k, probe_width=w, warp_sync=s, form=L.BATCH_PERSISTENT)
             for b in (128, 64, 256) for g in (1, 2, 4, 8) for k in (0, 2, 4) for s in (1, 0) for w in (1, 2)]
        return c[:max_candidates] if max_candidates > 0 else c

    def set_tuning(self, block=128, grab=2, smem_frames=0, probe_width=1, warp_sync=1, form=0) -> None:
        """form: L.BATCH_PERSISTENT (one persistent traversal launch per phase
        over all tables, tuned by the other fields) or L.BATCH_TABLE_GRAPHS (each
        table's own update kernels as concurrent branches of one graph)."""
        t = L.BatchTuning(block, grab, smem_frames, probe_width, warp_sync, form)
        L.check(self._lib.mccfr_batch_set_tuning(self._b, byref(t)))

    def tuning(self) -> dict:
        t = L.BatchTuning()
        L.check(self._lib.mccfr_batch_get_tuning(self._b, byref(t)))
        return t.as_dict()

    def stats(self) -> L.BatchStats:
        s = L.BatchStats()
        L.check(self._lib.mccfr_batch_get_stats(self._b, byref(s)))
        return s


def batch_round(trainers: list, traversals: list[int], tuning: dict | None = None) -> None:
    """One player-update of every listed trainer in one persistent launch
    (continuous batching step, mccfr_batch_round)."""
    lib = L.load()
    arr = (ctypes.c_void_p * len(trainers))(*[t.handle.value for t in trainers])
    cnt = (ctypes.c_int * len(traversals))(*[int(x) for x in traversals])
    tp = None
    if tuning:
        tp = byref(L.BatchTuning(tuning.get("block", 128), tuning.get("grab", 1), tuning.get("smem_frames", 0),
                                 tuning.get("probe_width", 1), tuning.get("warp_sync", 1)))
    L.check(lib.mccfr_batch_round(arr, len(trainers), cnt, tp))


def metrics_line(s0, s1, wall_s: float, iterations: int, batch: int) -> dict:
    """One JSON-lines record of a train() call from the stats before and after
    it: work counted on the device, rates over the call's wall time, and the
    kernels' CUDA-event times.  algorithmic_gbs is 40 B per node visit plus 96 B
    per updating-player update (key + regret row read; regret write, strategy
    row read and write) over the traversal kernels' time."""
    trav = s1.traversals - s0.traversals
    visits = s1.node_visits - s0.node_visits
    updates = s1.traverser_updates - s0.traverser_updates
    launches = max(1, s1.launches - s0.launches)
    tms = s1.traverse_ms - s0.traverse_ms
    ams = s1.apply_ms - s0.apply_ms
    return {
        "time": time.time(),
        "iteration": int(s1.iterations_done),
        "iterations": iterations,
        "traversals_per_update": batch,
        "wall_s": wall_s,
        "traversals": int(trav),
        "traversals_per_s": trav / wall_s if wall_s > 0 else None,
        "node_visits_per_s": visits / wall_s if wall_s > 0 else None,
        "hand_evals_per_s": (s1.hand_evals - s0.hand_evals) / wall_s if wall_s > 0 else None,
        "traverse_ms_per_update": tms / launches,
        "apply_ms_per_update": ams / launches,
        "algorithmic_gbs": (40.0 * visits + 96.0 * updates) / (tms / 1e3) / 1e9 if tms > 0 else None,
        "touched_rows_last_update": int(s1.touched_last),
        "device_error": int(s1.device_error),
    }

