"""Runs the reference's own GPU trainer (oracle/_ref/libref_gpu.so, built from
poker_cuda/src/cfr_gpu.cu unmodified) in a process of its own.

TEST INFRASTRUCTURE ONLY: tests/ and bench.py call it as a statistical checker
and as the reference's GPU timing; the product never loads it.  The reference
exits the process on a CUDA error (cfr_gpu.cu:61-69), which is why it runs here
and not inside the caller.

    python ref_gpu_run.py rows OUT_DIR PLAYERS ITERS BATCH TABLE_FILE
        trains GPUCFRTrainer(PLAYERS, 1000, 10, 20) and writes its non-zero rows:
        OUT_DIR/slots.npy (u32 FNV slots), regrets.npy and strategy_sum.npy
        ([rows][8] f32), plus OUT_DIR/info.json (num_info_sets_active, seconds)
    python ref_gpu_run.py time PLAYERS ITERS BATCH TABLE_FILE
        prints the reference's own summary line ("Done: ... hands/sec", the rate of
        its training loop, cfr_gpu.cu:1368-1377), then one JSON line with the
        rate of its benchmark mode for one fresh trainer: ITERS * BATCH * PLAYERS
        traversals over the wall time of the whole train() call (main.cpp:380-398)
"""
from __future__ import annotations

import ctypes
import json
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_ref" / "libref_gpu.so"
SLOTS = 1 << 26


def load() -> ctypes.CDLL:
    lib = ctypes.CDLL(str(LIB))
    lib.refgpu_create.restype = ctypes.c_void_p
    lib.refgpu_create.argtypes = [ctypes.c_int] * 4
    lib.refgpu_destroy.argtypes = [ctypes.c_void_p]
    lib.refgpu_load_hand_table.argtypes = [ctypes.c_void_p, ctypes.c_char_p]
    lib.refgpu_train.argtypes = [ctypes.c_void_p, ctypes.c_longlong, ctypes.c_int]
    lib.refgpu_export.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t]
    lib.refgpu_num_active.argtypes = [ctypes.c_void_p]
    return lib


def trainer(lib, players: int, table_file: str):
    h = lib.refgpu_create(players, 1000, 10, 20)
    if not lib.refgpu_load_hand_table(h, table_file.encode()):
        raise RuntimeError(f"the reference refused the table file {table_file}")
    return h


def main() -> int:
    mode = sys.argv[1]
    lib = load()
    if mode == "rows":
        out, players, iters, batch, table_file = Path(sys.argv[2]), *map(int, sys.argv[3:6]), sys.argv[6]
        h = trainer(lib, players, table_file)
        t0 = time.perf_counter()
        lib.refgpu_train(h, iters, batch)
        secs = time.perf_counter() - t0
        n = 8 * SLOTS
        r = np.empty(n, np.float32)
        s = np.empty(n, np.float32)
        assert lib.refgpu_export(h, r.ctypes.data, s.ctypes.data, n) == 1
        active = lib.refgpu_num_active(h)
        lib.refgpu_destroy(h)
        r = r.reshape(8, SLOTS)
        s = s.reshape(8, SLOTS)
        live = np.flatnonzero((r != 0).any(axis=0) | (s != 0).any(axis=0)).astype(np.uint32)
        out.mkdir(parents=True, exist_ok=True)
        np.save(out / "slots.npy", live)
        np.save(out / "regrets.npy", np.ascontiguousarray(r[:, live].T))
        np.save(out / "strategy_sum.npy", np.ascontiguousarray(s[:, live].T))
        (out / "info.json").write_text(json.dumps({"num_info_sets_active": active, "seconds": secs}))
        return 0
    if mode == "time":
        players, iters, batch, table_file = *map(int, sys.argv[2:5]), sys.argv[5]
        h = trainer(lib, players, table_file)
        t0 = time.perf_counter()
        lib.refgpu_train(h, iters, batch)
        secs = time.perf_counter() - t0
        libc = ctypes.CDLL(None)
        libc.fflush(None)  # the reference's own "Done: ... hands/sec" line, before ours
        lib.refgpu_destroy(h)
        print(json.dumps({"players": players, "iterations": iters, "batch": batch, "seconds": secs,
                          "traversals_per_s": iters * batch * players / secs}), flush=True)
        return 0
    raise SystemExit(f"unknown mode {mode}")


if __name__ == "__main__":
    sys.exit(main())
