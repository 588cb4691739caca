"""Subgame re-solve serving with continuous batching.

Requests are turn or river subgames (board, 2-6 players, pot, one 1326-combo
range per player, bet sizes, iteration budget).  The server keeps every admitted
request's regret table resident on the device and runs rounds: each round is
one mccfr_batch_round call, i.e. one player-update of every active request in a
single persistent traversal launch.  Requests that arrive while others run are
admitted between rounds as soon as a slot and device memory are free, and a
request retires (its strategy is copied to the host) as soon as its budget is
spent, so solves overlap on the device.  A request's result depends only on its
own tables and Philox keys, never on what it was batched with.
"""
from __future__ import annotations

import math
import threading
import time
from concurrent.futures import FIRST_COMPLETED, ThreadPoolExecutor
from concurrent.futures import wait as wait_futures
from dataclasses import dataclass, field

import numpy as np

from . import lib as L
from .trainer import GPUCFRTrainer, batch_round

# Bet sizes as pot fractions (num, den): 0.33, 0.5, 0.75, 1, 1.5, 2.
BET_SIZES = [(1, 3), (1, 2), (3, 4), (1, 1), (3, 2), (2, 1)]
CHIPS_PER_BB = 100
STACK_BB = 100


def combo_index(a: int, b: int) -> int:
    lo, hi = min(a, b), max(a, b)
    return hi * (hi - 1) // 2 + lo


def _combo_cards() -> np.ndarray:
    out = np.zeros((1326, 2), dtype=np.int64)
    for hi in range(1, 52):
        for lo in range(hi):
            out[combo_index(lo, hi)] = (lo, hi)
    return out


COMBO_CARDS = _combo_cards()


@dataclass
class Request:
    rid: int
    street: int                 # 2 turn, 3 river
    board: list[int]
    players: int
    pot: int                    # chips, a multiple of players
    ranges: np.ndarray          # [players][1326]
    sizes: list[tuple[int, int]]
    budget: int                 # traversals per player
    arrival: float = 0.0        # seconds since the start of the trace
    table_log2: int = 16


def make_request(rng: np.random.Generator, rid: int, max_sizes: int = 5) -> Request:
    """A request drawn as the re-solve workload specifies: uniform turn or river
    board, 2-6 players, pot U[2,200] BB, Dirichlet(0.5) ranges with board-blocked
    combos zeroed, 3-6 sizes from {0.33,0.5,0.75,1,1.5,2} pot plus all-in (at most
    `max_sizes`: fold, check/call, the sizes and all-in must fit 8 action
    slots), iteration budget log-uniform in [2e3, 5e4]."""
    street = int(rng.choice([2, 3]))
    players = int(rng.integers(2, 7))
    board = [int(c) for c in rng.permutation(52)[: (4 if street == 2 else 5)]]
    pot_bb = float(rng.uniform(2.0, 200.0))
    pot = max(players, int(round(pot_bb * CHIPS_PER_BB / players)) * players)
    blocked = np.isin(COMBO_CARDS, board).any(axis=1)
    ranges = rng.dirichlet(np.full(1326, 0.5), size=players).astype(np.float64)
    ranges[:, blocked] = 0.0
    ranges /= ranges.sum(axis=1, keepdims=True)
    k = int(rng.integers(3, 7))
    k = min(k, max_sizes)
    sizes = sorted(set(BET_SIZES[i] for i in rng.choice(6, size=k, replace=False)), key=lambda f: f[0] / f[1])
    budget = int(round(math.exp(rng.uniform(math.log(2e3), math.log(5e4)))))
    rows = budget * players * 64
    table_log2 = int(min(21, max(14, math.ceil(math.log2(max(rows, 2))))))
    return Request(rid, street, board, players, pot, ranges.astype(np.float32), sizes, budget,
                   table_log2=table_log2)


def request_config(req: Request) -> L.Config:
    c = L.preset(L.PRESET_HU_20BB)
    c.num_players = req.players
    c.small_blind = CHIPS_PER_BB // 2
    c.big_blind = CHIPS_PER_BB
    c.starting_stack = STACK_BB * CHIPS_PER_BB
    slots = [(L.ACT_FOLD, 0, 1), (L.ACT_CHECK_CALL, 0, 1)] + [(L.ACT_RAISE_POT, n, d) for n, d in req.sizes]
    slots.append((L.ACT_ALL_IN, 0, 1))
    c.num_actions = len(slots)
    for a, (k, n, d) in enumerate(slots):
        c.action_kind[a], c.action_num[a], c.action_den[a] = k, n, d
    c.raise_cap = 2
    c.max_depth = 255
    c.table_log2 = req.table_log2
    c.key_bits = req.table_log2 - 1
    c.seed = 0x5EED0000 + req.rid
    return c


def table_bytes(req: Request) -> int:
    """Device bytes of a request's table: 256-byte rows and a 4-byte touched-list
    entry per row, plus its small buffers."""
    return (1 << req.table_log2) * (256 + 4) + (1 << 20)


@dataclass
class Solve:
    req: Request
    trainer: GPUCFRTrainer
    updates_needed: int
    updates_done: int = 0
    admitted: float = 0.0


@dataclass
class Result:
    rid: int
    arrival: float
    admitted: float
    finished: float
    keys: np.ndarray = field(repr=False)
    probs: np.ndarray = field(repr=False)
    cancelled: bool = False     # withdrawn by cancel(): no strategy
    error: str = ""             # refused: the request can never be admitted (no strategy)

    @property
    def latency_ms(self) -> float:
        return (self.finished - self.arrival) * 1e3


class ReSolveServer:
    """Continuous-batching re-solver.

    hbm_budget: device bytes the server may hold in request tables, pooled ones
    included (admission also requires that much free device memory);
    max_active: requests batched per round (the persistent kernel takes up to 64
    tables); traversals: per player-update of each request.  Finished requests'
    tables are kept in a pool by capacity and reset for new requests of the
    same capacity (mccfr_subgame_reset), so a steady stream of requests
    allocates and frees no device memory; pooled tables are freed when a new
    capacity needs the room, and by close().

    cancel(rid), from any thread, withdraws a request: one not yet admitted is
    dropped, one being solved retires after the current round without exporting
    its strategy, and its table goes back to the pool.  A request that does not
    fit an idle server (its table above the budget, or above the free device
    memory with every pooled table freed) is refused with an error result
    instead of blocking the queue.  round_fn and create_fn
    replace the device round (batch_round) and the table creation, so the loop's
    host logic can run against stand-ins.

    retire_workers > 0 moves retiring off the round loop: a finished request's
    strategy is exported (a counting pass, a compaction and a copy on its own
    handle's stream, then the host sort) by a worker thread while the loop goes
    on running rounds for the others; its table counts against the budget until
    the export is done and then returns to the pool.  0 retires in the loop."""

    def __init__(self, rank_table_owner: GPUCFRTrainer, hbm_budget: int = 16 << 30, max_active: int = 64,
                 traversals: int = 256, tuning: dict | None = None, free_memory=None, round_fn=None,
                 create_fn=None, retire_workers: int = 0):
        self.owner = rank_table_owner
        self.hbm_budget = int(hbm_budget)
        self.max_active = min(64, int(max_active))
        self.traversals = int(traversals)
        self.tuning = tuning
        self.free_memory = free_memory or self._device_free
        self.rounds = 0
        # host seconds spent admitting (table creation), in rounds, and retiring
        self.timing = {"admit_s": 0.0, "round_s": 0.0, "retire_s": 0.0}
        self.pool: dict[int, list[GPUCFRTrainer]] = {}
        self.reused = 0
        self.cancelled = 0
        self.refused = 0
        self._round = round_fn or batch_round
        self._create = create_fn or self._create_subgame
        self._lock = threading.Lock()
        self._withdrawn: set[int] = set()
        self.retire_workers = int(retire_workers)

    def cancel(self, rid: int) -> None:
        with self._lock:
            self._withdrawn.add(int(rid))

    def _is_cancelled(self, rid: int) -> bool:
        with self._lock:
            return rid in self._withdrawn

    def _create_subgame(self, cfg: L.Config, req: Request) -> GPUCFRTrainer:
        t = GPUCFRTrainer.subgame(cfg, req.street, req.pot, req.board, req.ranges)
        t.share_hand_table(self.owner)
        return t

    @staticmethod
    def _device_free() -> int:
        import torch

        return int(torch.cuda.mem_get_info()[0])

    def pooled_bytes(self) -> int:
        return sum((1 << log2) * (256 + 4) + (1 << 20) for log2, ts in self.pool.items() for _ in ts)

    def _evict(self, need: int, held: int) -> None:
        """Frees pooled tables of other capacities until `need` more bytes fit."""
        for log2 in sorted(self.pool, key=lambda k: -k):
            while self.pool[log2] and held + self.pooled_bytes() + need > self.hbm_budget:
                self.pool[log2].pop().close()

    def admit_ok(self, req: Request, held: int, n_active: int) -> bool:
        if n_active >= self.max_active:
            return False
        if self.pool.get(req.table_log2):
            return True  # a pooled table of this capacity is reset, nothing is allocated
        need = table_bytes(req)
        self._evict(need, held)
        return held + self.pooled_bytes() + need <= self.hbm_budget and need + (1 << 30) <= self.free_memory()

    def _start(self, req: Request, now: float) -> Solve:
        cfg = request_config(req)
        ts = self.pool.get(req.table_log2)
        if ts:
            t = ts.pop()
            t.reset_subgame(cfg, req.street, req.pot, req.board, req.ranges)
            self.reused += 1
        else:
            t = self._create(cfg, req)
        return Solve(req, t, updates_for(req, self.traversals) * req.players, admitted=now)

    def close(self) -> None:
        """Frees the pooled tables."""
        for ts in self.pool.values():
            for t in ts:
                t.close()
        self.pool.clear()

    def run(self, requests: list[Request], realtime: bool = True) -> list[Result]:
        """Serves requests in arrival order; with realtime=False arrivals are
        ignored and every request is available at once."""
        pending = sorted(requests, key=lambda r: r.arrival)
        queue: list[Request] = []
        active: list[Solve] = []
        held = 0
        results: list[Result] = []
        t0 = time.perf_counter()
        none = np.zeros(0, np.uint32), np.zeros((0, 8), np.float32)

        def withdraw(req: Request, admitted: float) -> None:
            self.cancelled += 1
            results.append(Result(req.rid, req.arrival, admitted, time.perf_counter() - t0, *none, cancelled=True))

        def export(s: Solve):
            keys, probs = s.trainer.strategy_arrays()
            return keys, probs, time.perf_counter() - t0

        workers = ThreadPoolExecutor(self.retire_workers) if self.retire_workers > 0 else None
        retiring: list[tuple] = []  # (future, solve) of exports in flight

        def collect(wait: bool) -> int:
            """Books the exports that are done (waiting for one when `wait`);
            returns the device bytes their tables free for admission."""
            freed = 0
            if wait and retiring and not any(f.done() for f, _ in retiring):
                wait_futures([f for f, _ in retiring], return_when=FIRST_COMPLETED)
            for item in [x for x in retiring if x[0].done()]:
                f, s = item
                keys, probs, done_at = f.result()
                results.append(Result(s.req.rid, s.req.arrival, s.admitted, done_at, keys, probs))
                with self._lock:
                    self.pool.setdefault(s.req.table_log2, []).append(s.trainer)
                freed += table_bytes(s.req)
                retiring.remove(item)
            return freed

        try:
            self._serve(pending, queue, active, held, results, t0, none, withdraw, export, workers, retiring,
                        collect, realtime)
        finally:
            if workers is not None:
                workers.shutdown(wait=True)
        return results

    def _serve(self, pending, queue, active, held, results, t0, none, withdraw, export, workers, retiring, collect,
               realtime) -> None:
        while pending or queue or active or retiring:
            held -= collect(wait=False)
            now = time.perf_counter() - t0
            while pending and (not realtime or pending[0].arrival <= now):
                queue.append(pending.pop(0))
            for req in [r for r in queue if self._is_cancelled(r.rid)]:
                queue.remove(req)
                withdraw(req, now)
            ta = time.perf_counter()
            while queue and self.admit_ok(queue[0], held, len(active)):
                req = queue.pop(0)
                active.append(self._start(req, time.perf_counter() - t0))
                held += table_bytes(req)
            self.timing["admit_s"] += time.perf_counter() - ta
            if not active and retiring:
                held -= collect(wait=True)  # tables in export come back before anything is refused
                continue
            if not active and queue:
                # nothing runs and no pooled table is left to free, yet the head of
                # the queue does not fit: it never will, so it is refused rather
                # than left to block the requests behind it
                req = queue.pop(0)
                self.refused += 1
                results.append(Result(req.rid, req.arrival, now, time.perf_counter() - t0, *none,
                                      error=f"needs {table_bytes(req)} device bytes; budget {self.hbm_budget}, "
                                            f"free {self.free_memory()}"))
                continue
            if not active:
                if pending:
                    time.sleep(max(0.0, min(0.001, pending[0].arrival - now)))
                continue
            tr = time.perf_counter()
            self._round([s.trainer for s in active], [self.traversals] * len(active), self.tuning)
            self.rounds += 1
            tz = time.perf_counter()
            self.timing["round_s"] += tz - tr
            still = []
            for s in active:
                s.updates_done += 1
                if self._is_cancelled(s.req.rid):
                    withdraw(s.req, s.admitted)
                    self.pool.setdefault(s.req.table_log2, []).append(s.trainer)
                    held -= table_bytes(s.req)
                elif s.updates_done >= s.updates_needed:
                    if workers is not None:
                        retiring.append((workers.submit(export, s), s))  # its table is held until exported
                    else:
                        keys, probs, done_at = export(s)
                        results.append(Result(s.req.rid, s.req.arrival, s.admitted, done_at, keys, probs))
                        self.pool.setdefault(s.req.table_log2, []).append(s.trainer)  # kept for the next request
                        held -= table_bytes(s.req)
                else:
                    still.append(s)
            active[:] = still
            self.timing["retire_s"] += time.perf_counter() - tz


def updates_for(req: Request, traversals: int) -> int:
    """Player-updates a request's budget buys: the budget counts traversals per
    player (iterations of the one-traversal-per-player form), spent
    `traversals` at a time."""
    return max(1, math.ceil(req.budget / traversals))


def serve_plain(owner: GPUCFRTrainer, requests: list[Request], traversals: int = 256,
                realtime: bool = True) -> list[Result]:
    """The same requests on the plain trainer, one request at a time in arrival
    order: each is trained alone by `train` (one CUDA graph per iteration, every
    player-update of `traversals` traversals) until its budget is spent, then its
    strategy is copied out.  Tables are reused by capacity like the server's.
    The comparison point for continuous batching: same updates, same results."""
    pending = sorted(requests, key=lambda r: r.arrival)
    pool: dict[int, GPUCFRTrainer] = {}
    results: list[Result] = []
    t0 = time.perf_counter()
    try:
        for req in pending:
            now = time.perf_counter() - t0
            if realtime and req.arrival > now:
                time.sleep(req.arrival - now)
            admitted = time.perf_counter() - t0
            cfg = request_config(req)
            t = pool.get(req.table_log2)
            if t is None:
                t = GPUCFRTrainer.subgame(cfg, req.street, req.pot, req.board, req.ranges)
                t.share_hand_table(owner)
                pool[req.table_log2] = t
            else:
                t.reset_subgame(cfg, req.street, req.pot, req.board, req.ranges)
            t.train(updates_for(req, traversals), traversals, verbose=False)
            keys, probs = t.strategy_arrays()
            results.append(Result(req.rid, req.arrival, admitted, time.perf_counter() - t0, keys, probs))
    finally:
        for t in pool.values():
            t.close()
    return results


def poisson_arrivals(rng: np.random.Generator, n: int, rate: float) -> np.ndarray:
    return np.cumsum(rng.exponential(1.0 / rate, size=n))


def summarize(results: list[Result]) -> dict:
    """Latency percentiles and throughput of the solved requests; cancelled and
    refused ones are counted apart."""
    done = [r for r in results if not r.cancelled and not r.error]
    out = {"requests": len(done), "cancelled": sum(1 for r in results if r.cancelled),
           "refused": sum(1 for r in results if r.error)}
    if not done:
        return out
    lat = np.array([r.latency_ms for r in done])
    span = max(r.finished for r in done) - min(r.arrival for r in done)
    out.update({"p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                "mean_ms": float(lat.mean()), "solves_per_s": len(done) / span if span > 0 else None})
    return out
