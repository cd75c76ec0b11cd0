"""Builds the in-tree CUDA library ``libymkh.so`` for sm_100a.

The library is compiled with ``-fmad=false`` so that every FP64 product and
sum is rounded as written, which is what makes the step bit-comparable with
the reference kernels compiled the same way and with the FP64 CPU oracle.

Usage: ``python -m kh_simulations_b200.build [--force]``.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
INCLUDE = PKG.parent / "include"
LIB = PKG / "libymkh.so"

NVCC_FLAGS = [
    "-std=c++17",
    "-O3",
    "-lineinfo",
    "-fmad=false",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-shared",
    "-Xcompiler", "-fPIC",
    "-Xptxas", "-warn-spills",
]


def sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu"))


DEBUG_LIB = PKG / "libymkh_debug.so"


def _stale(lib: Path = LIB) -> bool:
    if not lib.exists():
        return True
    t = lib.stat().st_mtime
    deps = sources() + sorted(CSRC.glob("*.cuh")) + sorted(INCLUDE.glob("*.h"))
    return any(p.stat().st_mtime > t for p in deps)


def nvcc() -> str:
    cand = os.environ.get("NVCC") or "/usr/local/cuda/bin/nvcc"
    return cand if Path(cand).exists() else "nvcc"


def build(force: bool = False, verbose: bool = False, debug: bool = False) -> Path:
    """Compile csrc/*.cu into libymkh.so (skipped when up to date); with
    debug, into libymkh_debug.so with the kernels' access checks on
    (-DYMKH_DEBUG=1)."""
    lib = DEBUG_LIB if debug else LIB
    if not force and not _stale(lib):
        return lib
    cmd = [nvcc(), *NVCC_FLAGS, *(["-DYMKH_DEBUG=1"] if debug else []), f"-I{INCLUDE}", *map(str, sources()),
           "-o", str(lib)]
    if verbose:
        print(" ".join(cmd), flush=True)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed ({res.returncode}):\n{res.stderr}\n{res.stdout}")
    if verbose and res.stderr.strip():
        print(res.stderr, file=sys.stderr)
    return lib


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True, debug="--debug" in sys.argv))
