"""Builds libmccfr.so (sm_100a) in-tree, and the checker libraries under oracle/.

The product library is compiled with nvcc directly:
    nvcc -gencode arch=compute_100a,code=sm_100a -lineinfo -O3 -fmad=false ...
-fmad=false keeps every multiply and add separately rounded, as in the CPU
oracle (compiled with -ffp-contract=off), so sampled actions and table values
are bit-exact between the two.
"""
from __future__ import annotations

import os
import shutil
import subprocess
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB = PKG / "libmccfr.so"
ORACLE_DIR = ROOT / "oracle"

SOURCES = ["mccfr.cu", "eval_static.cu", "best_response.cu", "handtable.cpp", "abstraction.cpp"]
HEADERS = ["game.cuh", "table.cuh", "traverse_ref.cuh", "traverse_es.cuh", "traverse_levels.cuh", "showdown.cuh", "batched.cuh",
           "handtable.h", "best_response.h"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17", "-fmad=false",
    "-Xcompiler", "-fPIC", "-shared",
]


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps if d.exists())


def build_library(force: bool = False, verbose: bool = False) -> Path:
    deps = [CSRC / s for s in SOURCES + HEADERS] + [ROOT / "include" / "mccfr.h"]
    if not force and not _stale(LIB, deps):
        return LIB
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [_nvcc(), *NVCC_FLAGS, *[str(CSRC / s) for s in SOURCES], "-o", str(tmp)]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True, cwd=str(CSRC))
    os.replace(tmp, LIB)
    return LIB


CLI = PKG / "mccfr_cli"


def build_cli(force: bool = False) -> Path:
    """The command-line front end (reference flag names), linked to libmccfr.so."""
    deps = [CSRC / "cli.cpp", ROOT / "include" / "mccfr_trainer.hpp", ROOT / "include" / "mccfr.h", LIB]
    if not force and not _stale(CLI, deps):
        return CLI
    cuda_home = Path(_nvcc()).resolve().parent.parent
    cmd = ["g++", "-O2", "-std=c++17", str(CSRC / "cli.cpp"), f"-I{cuda_home / 'include'}", f"-L{PKG}", "-lmccfr",
           f"-L{cuda_home / 'lib64'}", "-lcudart", "-Wl,-rpath,$ORIGIN", f"-Wl,-rpath,{cuda_home / 'lib64'}",
           "-o", str(CLI)]
    subprocess.run(cmd, check=True)
    return CLI


def reference_sources_present() -> bool:
    """Whether oracle/Makefile finds the reference's sources (its REF directory,
    MCCFR_REFERENCE_SRC when set)."""
    r = subprocess.run(["make", "-s", "-C", str(ORACLE_DIR), "ref-check"], capture_output=True, text=True)
    return r.returncode == 0 and r.stdout.strip() == "yes"


def build_oracle(force: bool = False) -> Path:
    """Builds oracle/liboracle.so and, when the reference sources are present,
    oracle/_ref/libref.so (test infrastructure only)."""
    targets = ["all"]
    if reference_sources_present():
        targets.append("ref")
    cmd = ["make", "-s", "-C", str(ORACLE_DIR)]
    if force:
        cmd.append("-B")
    subprocess.run(cmd + targets, check=True)
    return ORACLE_DIR / "liboracle.so"


def build_all(force: bool = False, verbose: bool = False) -> None:
    build_library(force=force, verbose=verbose)
    build_cli(force=force)
    build_oracle(force=force)


if __name__ == "__main__":
    import sys

    build_all(force="--force" in sys.argv, verbose=True)
