"""The reference's own GPU trainer (poker_cuda/src/cfr_gpu.cu, compiled unchanged
for sm_100a into oracle/_ref/libref_gpu.so) against this trainer's reference
rule, statistically.  The reference draws from cuRAND, divides with fast math
and reads regrets while other threads add to them, so no bit-exact comparison
exists; what must agree is every property that does not depend on which random
numbers were drawn:

* its own 6-max game never learns (every player takes the passive fallback,
  24 decisions and 3 street changes reach the depth-20 cut, whose value is 0):
  all regrets stay exactly 0 in both, the touched slots average to the uniform
  strategy over their legal actions in both (all but the few slots that FNV
  collisions share between info sets of different legal masks, in equal
  shares), and the slots' visit counts (uniform deals through the same buckets
  and keys) agree within Poisson error;
* heads-up, where it learns: aggregate figures (touched slots, the strategy mass
  and positive-regret mass of each action slot) differ from this trainer's by
  no more than this trainer's own figures differ between seeds.

The reference runs in a child process (oracle/ref_gpu_run.py): it exits its
process on a CUDA error."""
from __future__ import annotations

import subprocess
import sys

import numpy as np
import pytest

from conftest import ROOT, mccfr

L = mccfr.lib
REF_GPU = ROOT / "oracle" / "_ref" / "libref_gpu.so"
pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not REF_GPU.exists(), reason="the reference's GPU trainer is not built here")]


def reference_rows(tmp_path, table_file, players, iters, batch):
    out = tmp_path / f"ref_{players}_{iters}_{batch}"
    subprocess.run([sys.executable, str(ROOT / "oracle" / "ref_gpu_run.py"), "rows", str(out), str(players),
                    str(iters), str(batch), str(table_file)], check=True, timeout=900)
    return {"slots": np.load(out / "slots.npy"), "regrets": np.load(out / "regrets.npy"),
            "strategy_sum": np.load(out / "strategy_sum.npy")}


def our_rows(table, players, iters, batch, seed=42):
    cfg = L.preset(L.PRESET_REF8)
    cfg.num_players, cfg.seed = players, seed
    t = mccfr.GPUCFRTrainer(config=cfg)
    t.set_hand_table(table)
    t.train(iters, batch, verbose=False)
    r = t.export_rows()
    t.close()
    live = (r["regrets"] != 0).any(1) | (r["strategy_sum"] != 0).any(1)
    return {"slots": (r["keys"][live] - 1).astype(np.uint32), "regrets": r["regrets"][live],
            "strategy_sum": r["strategy_sum"][live]}


def uniform_share(ssum):
    """Fraction of rows whose non-zero strategy sums are all equal: a uniform
    average strategy.  A slot shared by info sets with different legal masks (an
    FNV collision) sums different uniform strategies, so a few rows are not."""
    s = ssum.astype(np.float64)
    hi = np.where(s > 0, s, -np.inf).max(1)
    lo = np.where(s > 0, s, np.inf).min(1)
    assert np.all(s >= 0)
    return float(np.mean((hi - lo) <= 1e-5 * hi))


def test_reference_six_max_never_learns_in_either(hand_table, hand_table_file, tmp_path):
    batch = 1 << 18
    ref = reference_rows(tmp_path, hand_table_file, 6, 1, batch)
    ours = our_rows(hand_table, 6, 1, batch)
    shares = []
    for d in (ref, ours):
        assert np.all(d["regrets"] == 0)
        shares.append(uniform_share(d["strategy_sum"]))
    assert min(shares) > 0.99 and abs(shares[0] - shares[1]) < 0.002, shares
    # one iteration, weight 1: a slot's strategy sum is its visit count
    ca = dict(zip(ref["slots"].tolist(), ref["strategy_sum"].sum(1).round().astype(np.int64).tolist()))
    cb = dict(zip(ours["slots"].tolist(), ours["strategy_sum"].sum(1).round().astype(np.int64).tolist()))
    assert abs(sum(ca.values()) - sum(cb.values())) <= 5 * np.sqrt(sum(ca.values()))
    heavy = [s for s in set(ca) | set(cb) if ca.get(s, 0) + cb.get(s, 0) >= 200]
    assert len(heavy) > 1000
    a = np.array([ca.get(s, 0) for s in heavy], np.float64)
    b = np.array([cb.get(s, 0) for s in heavy], np.float64)
    z = (a - b) / np.sqrt(a + b)
    assert abs(z.mean()) < 0.1 and 0.8 < z.std() < 1.25, (z.mean(), z.std())
    assert np.mean(np.abs(z) > 5) < 1e-3
    # a slot with many visits in one is visited in the other
    assert all(s in ca and s in cb for s in heavy if ca.get(s, 0) >= 100 or cb.get(s, 0) >= 100)


def aggregates(d):
    s = d["strategy_sum"].astype(np.float64).sum(0)
    r = np.maximum(d["regrets"].astype(np.float64), 0).sum(0)
    return d["slots"].size, s / s.sum(), r / max(r.sum(), 1e-30)


def test_reference_heads_up_agrees_within_seed_noise(hand_table, hand_table_file, tmp_path):
    iters, batch = 2, 1 << 16
    ref = aggregates(reference_rows(tmp_path, hand_table_file, 2, iters, batch))
    mine = [aggregates(our_rows(hand_table, 2, iters, batch, seed)) for seed in (42, 43, 44)]
    n_noise = max(abs(x[0] - y[0]) for x in mine for y in mine)
    assert abs(ref[0] - mine[0][0]) <= 4 * n_noise + 0.002 * mine[0][0], (ref[0], [m[0] for m in mine])
    for k in (1, 2):
        noise = np.max([np.abs(x[k] - y[k]) for x in mine for y in mine], axis=0)
        diff = np.abs(ref[k] - mine[0][k])
        assert np.all(diff <= 4 * noise + 2e-3), (k, diff, noise)
