"""The multi-rank path of bench.py on CPU: two gloo ranks, world size 2.

`bench.py --gpus N` runs N independent replicas, one per rank, with no
data-path collective; only the figures are combined.  Here each rank runs a
small replica on the CPU oracle in place of the device trainer.  The test checks
that the ranks' seeds differ, that their tables differ, and that `over_ranks`
gives the slowest rank's times and the sum of all ranks' traversals, the same
figures on every rank."""
from __future__ import annotations

import json
import os
import socket
import sys
import time
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
WORLD = 2
BATCH = 256


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, port: int, table_path: str, out_dir: str) -> None:
    sys.path[:0] = [str(ROOT), str(ROOT / "oracle")]
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(WORLD))
    from datetime import timedelta

    import torch.distributed as dist

    import __graft_entry__ as ge
    import bench
    import binding

    dist.init_process_group("gloo", rank=rank, world_size=WORLD, timeout=timedelta(seconds=60))
    try:
        L = ge.load_package().lib
        cfg, _ = bench.make_config(L, "hu-20bb", rank)
        cfg.table_log2, cfg.key_bits = 16, 15
        orc = binding.Oracle(cfg, np.fromfile(table_path, dtype=np.int32))
        t0 = time.perf_counter()
        for p in range(cfg.num_players):
            orc.step(1, p, BATCH * (rank + 1), threads=1)  # ranks do unequal work
        ms = (time.perf_counter() - t0) * 1e3
        trav = BATCH * (rank + 1) * cfg.num_players
        e2e_s = 0.5 + rank  # stands in for the rank's host-timed loop
        rows = orc.export_rows()
        digest = int(np.bitwise_xor.reduce(rows["keys"].view(np.uint64))) if rows["keys"].size else 0
        orc.close()

        got = bench.over_ranks(ms, trav, e2e_s, "cpu")
        mine = {"rank": rank, "seed": int(cfg.seed), "ms": ms, "trav": trav, "e2e_s": e2e_s,
                "rows": int(rows["keys"].size), "digest": digest, "got": got}
        every = [None] * WORLD
        dist.all_gather_object(every, mine)
        if rank == 0:
            Path(out_dir, "ranks.json").write_text(json.dumps(every))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_over_ranks_without_process_group():
    sys.path.insert(0, str(ROOT))
    import bench

    assert bench.over_ranks(12.5, 4096, 3.0, "cpu") == (12.5, 4096.0, 3.0)


def test_two_gloo_replicas(hand_table_file, tmp_path):
    import torch.multiprocessing as mp

    mp.spawn(_rank_main, args=(_free_port(), str(hand_table_file), str(tmp_path)), nprocs=WORLD, join=True)
    ranks = json.loads((tmp_path / "ranks.json").read_text())
    assert [r["rank"] for r in ranks] == list(range(WORLD))
    assert len({r["seed"] for r in ranks}) == WORLD
    assert all(r["rows"] > 0 for r in ranks)
    assert ranks[0]["digest"] != ranks[1]["digest"]  # independent replicas, not copies
    want = (max(r["ms"] for r in ranks), float(sum(r["trav"] for r in ranks)), max(r["e2e_s"] for r in ranks))
    for r in ranks:
        assert r["got"] == pytest.approx(list(want), rel=1e-12)
    assert want[1] == BATCH * 2 * (1 + 2)
