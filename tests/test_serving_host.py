"""Host logic of the re-solve server (CPU): request generation and admission."""
from __future__ import annotations

import importlib
import time

import numpy as np
import pytest

from conftest import mccfr  # noqa: F401  (registers mccfr_b200)

sv = importlib.import_module("mccfr_b200.serving")


def test_requests_follow_the_workload():
    rng = np.random.default_rng(0)
    for rid in range(200):
        r = sv.make_request(rng, rid)
        assert r.street in (2, 3) and len(r.board) == (4 if r.street == 2 else 5)
        assert len(set(r.board)) == len(r.board)
        assert 2 <= r.players <= 6 and r.pot % r.players == 0
        assert 2 * 100 - r.players <= r.pot <= 200 * 100 + r.players
        assert r.ranges.shape == (r.players, 1326)
        blocked = np.isin(sv.COMBO_CARDS, r.board).any(axis=1)
        assert np.all(r.ranges[:, blocked] == 0)
        assert np.allclose(r.ranges.sum(1), 1.0, atol=1e-5)
        assert 3 <= len(r.sizes) <= 5 and all(s in sv.BET_SIZES for s in r.sizes)
        assert 2000 <= r.budget <= 50000
        assert 14 <= r.table_log2 <= 21
        c = sv.request_config(r)
        assert c.num_actions == len(r.sizes) + 3 <= 8


def test_combo_index_is_a_bijection():
    seen = {sv.combo_index(a, b) for a in range(52) for b in range(a + 1, 52)}
    assert seen == set(range(1326))
    for i, (lo, hi) in enumerate(sv.COMBO_CARDS):
        assert sv.combo_index(lo, hi) == i


def test_admission_respects_budget_and_free_memory():
    rng = np.random.default_rng(1)
    req = sv.make_request(rng, 0)
    need = sv.table_bytes(req)
    srv = sv.ReSolveServer(None, hbm_budget=3 * need, max_active=2, free_memory=lambda: 100 << 30)
    assert srv.admit_ok(req, 0, 0)
    assert not srv.admit_ok(req, 0, 2)          # slots
    assert not srv.admit_ok(req, 3 * need, 0)   # budget
    tight = sv.ReSolveServer(None, hbm_budget=1 << 40, free_memory=lambda: need)
    assert not tight.admit_ok(req, 0, 0)        # device memory


def test_poisson_arrivals_rate():
    rng = np.random.default_rng(2)
    a = sv.poisson_arrivals(rng, 20000, 100.0)
    assert np.all(np.diff(a) > 0)
    assert abs(20000 / a[-1] - 100.0) < 3.0


class _FakeTrainer:
    def __init__(self):
        self.closed = False

    def close(self):
        self.closed = True


def test_pool_reuse_and_eviction():
    """A pooled table of the request's capacity is reused with nothing
    allocated; tables of other capacities are freed when room is needed."""
    rng = np.random.default_rng(3)
    req = sv.make_request(rng, 0)
    need = sv.table_bytes(req)
    srv = sv.ReSolveServer(None, hbm_budget=2 * need, free_memory=lambda: 100 << 30)
    same = _FakeTrainer()
    srv.pool[req.table_log2] = [same]
    assert srv.admit_ok(req, 2 * need, 0)        # full budget, but the pooled table is reused
    other = _FakeTrainer()
    other_log2 = req.table_log2 - 1 if req.table_log2 > 14 else req.table_log2 + 1
    srv.pool = {other_log2: [other]}
    assert srv.admit_ok(req, need, 0)             # the other-capacity table is freed to make room
    assert other.closed and not srv.pool[other_log2]
    srv.pool = {other_log2: [_FakeTrainer()]}
    assert not srv.admit_ok(req, 2 * need, 0)     # no room even with the pool empty
    srv.close()
    assert srv.pool == {}


class _FakeSolver:
    """Stands in for a subgame trainer: counts its rounds and resets."""

    def __init__(self):
        self.closed = False
        self.rounds = 0
        self.resets = 0

    def reset_subgame(self, *args):
        self.resets += 1
        self.rounds = 0

    def strategy_arrays(self):
        return np.array([7], np.uint32), np.full((1, 8), 0.125, np.float32)

    def close(self):
        self.closed = True


def _same_size_requests(n: int) -> list:
    rng = np.random.default_rng(5)
    reqs = [sv.make_request(rng, rid) for rid in range(n)]
    for r in reqs:
        r.table_log2, r.budget, r.players = 16, 4 * 256, 2  # 4 rounds per player, 8 rounds each
    return reqs


def test_cancel_before_admission_and_mid_solve():
    """A request withdrawn while queued never gets a table; one withdrawn
    mid-solve retires after that round with no strategy, and its table is reused
    by the next request.  The others finish with their full budgets."""
    reqs = _same_size_requests(4)
    made = []
    rounds = [0]

    def create(cfg, req):
        made.append(_FakeSolver())
        return made[-1]

    def round_fn(trainers, traversals, tuning):
        rounds[0] += 1
        for t in trainers:
            t.rounds += 1
        if rounds[0] == 3:
            srv.cancel(reqs[0].rid)  # a client withdraws mid-solve

    need = sv.table_bytes(reqs[0])
    srv = sv.ReSolveServer(None, hbm_budget=4 * need, max_active=2, free_memory=lambda: 100 << 30,
                           traversals=256, round_fn=round_fn, create_fn=create)
    srv.cancel(reqs[3].rid)  # withdrawn before it is admitted
    res = {r.rid: r for r in srv.run(reqs, realtime=False)}
    assert set(res) == {r.rid for r in reqs}
    assert res[reqs[0].rid].cancelled and res[reqs[0].rid].keys.size == 0
    assert res[reqs[3].rid].cancelled
    for r in (reqs[1], reqs[2]):
        assert not res[r.rid].cancelled and res[r.rid].keys.tolist() == [7]
    assert srv.cancelled == 2
    # two tables were made; request 2 ran on request 0's returned table
    assert len(made) == 2 and srv.reused == 1
    assert made[0].resets == 1
    srv.close()
    assert all(t.closed for t in made)


def test_cancel_from_another_thread_is_safe():
    import threading

    reqs = _same_size_requests(3)
    started, withdrawn = threading.Event(), threading.Event()

    def round_fn(trainers, traversals, tuning):
        if not started.is_set():
            started.set()
            assert withdrawn.wait(5)  # the first round ends after the other thread's cancel
        for t in trainers:
            t.rounds += 1

    def client():
        assert started.wait(5)
        srv.cancel(reqs[2].rid)
        withdrawn.set()

    srv = sv.ReSolveServer(None, hbm_budget=1 << 40, max_active=1, free_memory=lambda: 100 << 30,
                           traversals=256, round_fn=round_fn, create_fn=lambda cfg, req: _FakeSolver())
    th = threading.Thread(target=client)
    th.start()
    res = {r.rid: r for r in srv.run(reqs, realtime=False)}
    th.join()
    assert res[reqs[2].rid].cancelled  # still queued behind the single slot when withdrawn
    assert not res[reqs[0].rid].cancelled and not res[reqs[1].rid].cancelled


def test_summary_leaves_out_cancelled_requests():
    e = (np.zeros(0, np.uint32), np.zeros((0, 8), np.float32))
    res = [sv.Result(0, 0.0, 0.0, 0.1, *e), sv.Result(1, 0.0, 0.0, 0.3, *e),
           sv.Result(2, 0.0, 0.0, 9.0, *e, cancelled=True)]
    s = sv.summarize(res)
    assert s["requests"] == 2 and s["cancelled"] == 1
    assert s["p50_ms"] == pytest.approx(200.0) and s["mean_ms"] == pytest.approx(200.0)
    assert sv.summarize(res[2:]) == {"requests": 0, "cancelled": 1, "refused": 0}


def test_request_that_can_never_fit_is_refused_not_spun_on():
    """A request whose table exceeds the whole budget, at the head of the queue
    of an idle server, is refused with an error result (the loop used to retry
    it forever); the requests behind it are served."""
    reqs = _same_size_requests(3)
    big = reqs[0]
    big.table_log2 = 21
    need_small = sv.table_bytes(reqs[1])
    assert sv.table_bytes(big) > 4 * need_small

    def round_fn(trainers, traversals, tuning):
        for t in trainers:
            t.rounds += 1

    srv = sv.ReSolveServer(None, hbm_budget=4 * need_small, max_active=2, free_memory=lambda: 100 << 30,
                           traversals=256, round_fn=round_fn, create_fn=lambda cfg, req: _FakeSolver())
    res = {r.rid: r for r in srv.run(reqs, realtime=False)}
    assert res[big.rid].error and "device bytes" in res[big.rid].error and res[big.rid].keys.size == 0
    for r in reqs[1:]:
        assert not res[r.rid].error and res[r.rid].keys.tolist() == [7]
    assert srv.refused == 1
    s = sv.summarize(list(res.values()))
    assert s["requests"] == 2 and s["refused"] == 1


def test_device_memory_short_of_a_request_refuses_it():
    """Free device memory below a request's table (plus the 1 GiB reserve) with
    nothing running: refused the same way."""
    reqs = _same_size_requests(1)
    srv = sv.ReSolveServer(None, hbm_budget=1 << 40, free_memory=lambda: 1 << 20, traversals=256,
                           round_fn=lambda *a: None, create_fn=lambda cfg, req: _FakeSolver())
    res = srv.run(reqs, realtime=False)
    assert len(res) == 1 and res[0].error


def test_budget_counts_traversals_per_player():
    reqs = _same_size_requests(1)
    assert sv.updates_for(reqs[0], 256) == 4
    reqs[0].budget = 1000
    assert sv.updates_for(reqs[0], 256) == 4  # rounded up


def test_retire_workers_export_while_rounds_go_on():
    """With a retire worker a finished request's export runs beside the rounds of
    the others: rounds happen while an export is in flight, every request still
    gets its strategy, and the exported tables return to the pool for reuse."""
    import threading

    reqs = _same_size_requests(4)
    reqs[0].budget = 256  # finishes after one round per player, long before the others
    exporting = threading.Event()
    rounds_while_exporting = [0]

    class SlowExport(_FakeSolver):
        def strategy_arrays(self):
            exporting.set()
            time.sleep(0.2)
            exporting.clear()
            return super().strategy_arrays()

    def round_fn(trainers, traversals, tuning):
        if exporting.is_set():
            rounds_while_exporting[0] += 1
        time.sleep(0.01)

    # room for three tables: the fourth request waits for an exported table
    srv = sv.ReSolveServer(None, hbm_budget=3 * sv.table_bytes(reqs[0]), max_active=3,
                           free_memory=lambda: 100 << 30, traversals=256, round_fn=round_fn,
                           create_fn=lambda cfg, req: SlowExport(), retire_workers=1)
    res = {r.rid: r for r in srv.run(reqs, realtime=False)}
    assert set(res) == {r.rid for r in reqs}
    assert all(r.keys.tolist() == [7] and not r.error and not r.cancelled for r in res.values())
    assert rounds_while_exporting[0] > 0
    assert srv.reused >= 1  # the fourth request ran on the table that came back from an export
    srv.close()
