"""Brute-force heads-up best response for small subgames (checker of the
library's vector best response, mccfr_best_response).

TEST INFRASTRUCTURE ONLY: imported by tests/ as the checker, never by the
product.  Independent of the library's engine in every step that matters: the
betting tree is replayed here from the traversal's rules (valid_mask and
chips_for through the oracle library, the state update of es_apply restated in
Python), info-set keys are recomputed in Python, each of the best responder's
combos is walked on its own with an explicit opponent distribution, and every
showdown compares the two 7-card ranks pair by pair.  Only practical for
ranges of a few combos.
"""
from __future__ import annotations

import ctypes

import numpy as np

try:
    from . import binding as B
except ImportError:  # imported as a top-level module (tests put oracle/ on sys.path)
    import binding as B

M64 = (1 << 64) - 1
PATH_SEED = 0x243F6A8885A308D3


def path_step(h: int, a: int) -> int:
    h = ((h ^ (a + 1)) * 0x9E3779B97F4A7C15) & M64
    return h ^ (h >> 31)


def mix64(z: int) -> int:
    z ^= z >> 33
    z = (z * 0xFF51AFD7ED558CCD) & M64
    z ^= z >> 33
    z = (z * 0xC4CEB9FE1A85EC53) & M64
    z ^= z >> 33
    return z


def info_key(player: int, hb: int, bb: int, street: int, path: int, key_bits: int) -> int:
    k = path ^ (player << 56) ^ (hb << 44) ^ (bb << 32) ^ (street << 28)
    k = mix64(k & M64)
    if key_bits > 0:
        return (k & ((1 << key_bits) - 1)) + 1
    return k if k else 1


def combo_cards(c: int) -> tuple[int, int]:
    hi = 1
    while (hi + 1) * hi // 2 <= c:
        hi += 1
    return c - hi * (hi - 1) // 2, hi


class Game:
    """A heads-up subgame: betting rules from the config, root as the trainer's."""

    def __init__(self, cfg, street: int, pot: int, board, weights: np.ndarray, table: np.ndarray):
        self.cfg = cfg
        self.street0 = street
        self.pot0 = pot
        self.board = list(board)[: 4 if street == 2 else 5]
        self.w = weights  # [2][1326] quantised weights
        self.T = table
        self.kind = [cfg.action_kind[a] if a < cfg.num_actions else -1 for a in range(8)]
        self._rank = {}

    def rank(self, cards) -> int:
        key = tuple(sorted(cards))
        r = self._rank.get(key)
        if r is None:
            r = int(B.eval7(self.T, np.array([key], dtype=np.uint8))[0])
            self._rank[key] = r
        return r

    def root(self) -> dict:
        g = self.cfg
        return dict(stack=[g.starting_stack] * 2, bet=[0, 0], inv=[self.pot0 // 2] * 2, pot=self.pot0, cb=0,
                    lfr=g.big_blind, q=[0, 1], folded=[False, False], allin=[False, False], street=self.street0,
                    raises=0, depth=0, path=PATH_SEED)

    def legal(self, s) -> list[int]:
        p = s["q"][0]
        vm = B.valid_mask(self.cfg, s["pot"], s["stack"][p], s["cb"] - s["bet"][p], s["cb"], s["lfr"], s["raises"])
        return [a for a in range(8) if (vm >> a) & 1]

    def apply(self, s, a) -> dict:
        s = {k: (list(v) if isinstance(v, list) else v) for k, v in s.items()}
        p = s["q"].pop(0)
        to_call = s["cb"] - s["bet"][p]
        chips = B.chips(self.cfg, a, s["pot"], s["stack"][p], to_call, s["cb"], s["lfr"])
        s["path"] = path_step(s["path"], a)
        k = self.kind[a]
        if k == 0:
            s["folded"][p] = True
            return s
        if k == 1:
            return s
        s["stack"][p] -= chips
        s["bet"][p] += chips
        s["inv"][p] += chips
        s["pot"] += chips
        if s["stack"][p] == 0:
            s["allin"][p] = True
        if s["bet"][p] > s["cb"]:
            prev = s["cb"]
            rs = s["bet"][p] - prev
            if rs >= s["lfr"] or prev == 0:
                s["lfr"] = rs
            s["cb"] = s["bet"][p]
            s["raises"] += 1
            o = 1 - p
            s["q"] = [] if (s["folded"][o] or s["allin"][o]) else [o]
        return s

    def next_street(self, s) -> dict:
        s = {k: (list(v) if isinstance(v, list) else v) for k, v in s.items()}
        s["street"] += 1
        s["bet"] = [0, 0]
        s["cb"] = 0
        s["lfr"] = self.cfg.big_blind
        s["raises"] = 0
        s["q"] = [p for p in (0, 1) if not s["folded"][p] and not s["allin"][p]]  # dealer is seat 1
        return s


def payoff(s, i: int, ranks) -> float:
    """Net chips of player i at a showdown (heads-up side_pot_payoff)."""
    inv = s["inv"]
    m = min(inv)
    if ranks[0] == ranks[1]:
        return 0.0
    win = 0 if ranks[0] > ranks[1] else 1
    return float(m) if win == i else -float(m)


def strategy(rows: dict, g: Game, s, player: int, combo: int, river: int) -> dict:
    legal = g.legal(s)
    bkt = river + 1 if (s["street"] == 3 and g.street0 == 2) else 0
    key = info_key(player, combo, bkt, s["street"], s["path"], g.cfg.key_bits)
    row = rows.get(key)
    tot = sum(max(0.0, float(row[a])) for a in legal) if row is not None else 0.0
    if row is None or tot <= 0.0:
        return {a: 1.0 / len(legal) for a in legal}
    return {a: max(0.0, float(row[a])) / tot for a in legal}


def _value(g: Game, rows: dict, s, i: int, ci: int, dist: dict, river: int) -> float:
    """Best-response value of player i holding ci; dist maps the opponent's
    combos to their weight (range x its strategy along the path)."""
    cfg = g.cfg
    if s["depth"] >= cfg.max_depth:
        return 0.0
    live = [p for p in (0, 1) if not s["folded"][p]]
    if len(live) == 1:
        w = live[0]
        pay = (s["pot"] - s["inv"][i]) if w == i else -s["inv"][i]
        return pay * sum(dist.values())
    if not s["q"]:
        if s["street"] < 3:
            t = g.next_street(s)
            if t["q"]:
                t["depth"] += 1
                return _deal(g, rows, t, i, ci, dist, river, lambda u, d, r: _value(g, rows, u, i, ci, d, r))
            return _deal(g, rows, t, i, ci, dist, river, lambda u, d, r: _showdown(g, u, i, ci, d, r))
        return _showdown(g, s, i, ci, dist, river)
    p = s["q"][0]
    legal = g.legal(s)
    if p == i:
        best = None
        for a in legal:
            t = g.apply(s, a)
            t["depth"] += 1
            v = _value(g, rows, t, i, ci, dist, river)
            best = v if best is None else max(best, v)
        return best
    total = 0.0
    for a in legal:
        nd = {}
        for co, w in dist.items():
            pa = strategy(rows, g, s, p, co, river)[a]
            if pa > 0.0 and w > 0.0:
                nd[co] = w * pa
        t = g.apply(s, a)
        t["depth"] += 1
        total += _value(g, rows, t, i, ci, nd, river)
    return total


def _deal(g: Game, rows: dict, s, i: int, ci: int, dist: dict, river: int, cont) -> float:
    """The river card (turn subgames): 44 cards fit any pair of hands."""
    if s["street"] != 3 or g.street0 == 3:
        return cont(s, dist, river)
    lo, hi = combo_cards(ci)
    total = 0.0
    for r in range(52):
        if r in g.board or r in (lo, hi):
            continue
        nd = {co: w for co, w in dist.items() if r not in combo_cards(co)}
        total += cont(s, nd, r) / 44.0
    return total


def _showdown(g: Game, s, i: int, ci: int, dist: dict, river: int) -> float:
    board = g.board + ([river] if g.street0 == 2 else [])
    lo, hi = combo_cards(ci)
    ri = g.rank(board + [lo, hi])
    total = 0.0
    for co, w in dist.items():
        a, b = combo_cards(co)
        ro = g.rank(board + [a, b])
        ranks = (ri, ro) if i == 0 else (ro, ri)
        total += w * payoff(s, i, ranks)
    return total


def best_response_values(cfg, street: int, pot: int, board, ranges: np.ndarray, table: np.ndarray,
                         keys: np.ndarray, ssum: np.ndarray) -> tuple[float, float]:
    """(br_value[0], br_value[1]) in chips per game, by brute force."""
    board = list(board)
    nb = 4 if street == 2 else 5
    bmask = 0
    for c in board[:nb]:
        bmask |= 1 << c
    w = np.zeros((2, 1326), dtype=np.float64)
    for p in range(2):
        r = np.ascontiguousarray(ranges[p], dtype=np.float32)
        cdf = np.zeros(1326, dtype=np.uint32)
        bd = np.zeros(5, dtype=np.uint8)
        bd[:nb] = board[:nb]
        assert B.lib().orc_range_cdf(B._p(r), B._p(bd), nb, B._p(cdf)) == 1
        prev = np.concatenate([[0], cdf[:-1].astype(np.float64)])
        w[p] = cdf.astype(np.float64) - prev
    g = Game(cfg, street, pot, board, w, table)
    rows = {int(k): ssum[j] for j, k in enumerate(keys)}
    Z = 0.0
    combos = [[c for c in range(1326) if w[p][c] > 0] for p in range(2)]
    for c0 in combos[0]:
        m0 = set(combo_cards(c0))
        for c1 in combos[1]:
            if not (m0 & set(combo_cards(c1))):
                Z += w[0][c0] * w[1][c1]
    out = []
    for i in range(2):
        o = 1 - i
        total = 0.0
        for ci in combos[i]:
            mi = set(combo_cards(ci))
            dist = {co: w[o][co] for co in combos[o] if not (mi & set(combo_cards(co)))}
            if not dist:
                continue
            total += w[i][ci] * _value(g, rows, g.root(), i, ci, dist, -1)
        out.append(total / Z)
    return out[0], out[1]
