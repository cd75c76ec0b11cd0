"""Readers for the state snapshots written by ``KHRun.snapshot`` /
``ymkh_snapshot`` (include/ymkh.h).

- ``read_fp64``: the exact binary form (40-byte header "YMKHSNP1", then the
  24 arrays in state order).
- ``read_csv``: the reference's 26-column CSV (ymgpu2d/main_ym.cu:287-306),
  as the reference's analysis scripts read it (they reshape each column to
  [NZ, NX], e.g. ymgpu2d/analysis/gauss_check.py:44-45).
"""
from __future__ import annotations

import struct
from pathlib import Path

import numpy as np

from ._lib import NSTATE

MAGIC = b"YMKHSNP1"
CSV_COLUMNS = ("X", "Z", "By1", "By2", "By3", "Az2", "Az3", "PzA", "PxA", "Q1A", "PzB", "PxB", "Q1B",
               "Ex1", "Ex2", "Ex3", "Ez1", "Ez2", "Ez3", "nA", "nB", "Q2A", "Q3A", "Q2B", "Q3B", "Az1")


def read_fp64(path: str | Path) -> tuple[np.ndarray, float, float]:
    """(state [24, NZ, NX] float64, dx, dz) of an FP64 snapshot."""
    raw = Path(path).read_bytes()
    if raw[:8] != MAGIC:
        raise ValueError(f"{path}: not an FP64 snapshot")
    version, nx, nz, narr = struct.unpack_from("<4I", raw, 8)
    dx, dz = struct.unpack_from("<2d", raw, 24)
    if version != 1 or narr != NSTATE:
        raise ValueError(f"{path}: version {version}, {narr} arrays")
    n = NSTATE * nx * nz
    if len(raw) != 40 + 8 * n:
        raise ValueError(f"{path}: {len(raw)} bytes, expected {40 + 8 * n}")
    st = np.frombuffer(raw, dtype="<f8", count=n, offset=40).reshape(NSTATE, nz, nx).copy()
    return st, dx, dz


def read_csv(path: str | Path) -> dict:
    """Columns of a 26-column CSV snapshot, each [NZ, NX]; NX is the number
    of rows before Z first changes."""
    with open(path) as fh:
        header = fh.readline().strip().split(",")
    if tuple(header) != CSV_COLUMNS:
        raise ValueError(f"{path}: unexpected header {header[:4]}...")
    data = np.loadtxt(path, delimiter=",", skiprows=1, ndmin=2)
    z = data[:, 1]
    nx = int(np.argmax(z != z[0])) or len(z)
    nz = len(z) // nx
    return {c: data[:, i].reshape(nz, nx) for i, c in enumerate(CSV_COLUMNS)}
