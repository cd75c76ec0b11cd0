"""Eigenmode seed profiles: the reference's ``.bin`` format and its float
interpolation to the grid.

File format (ymgpu2d/main_ym.cu:179-181, written by
ymgpu2d/analysis/ym_eigenmode.py:411-440): ``int32 n_fields``, ``int32
nx_file``, then ``n_fields * nx_file`` float32 values, field-major, in the
order by, ex, ez, az, qA, qB.  At most six fields are used.

``interpolate`` repeats ymgpu2d/main_ym.cu:198-206 in float32 arithmetic:
``t = i*(float)(nx_file-1)/(float)(NX-1)``, ``j = min((int)t, nx_file-2)``,
``frc = t - j``, ``h[j]*(1-frc) + h[j+1]*frc``, then widened to double.
"""
from __future__ import annotations

import struct
from pathlib import Path

import numpy as np

FIELD_ORDER = ("by", "ex", "ez", "az", "qA", "qB")


class SeedError(ValueError):
    pass


def read_seed(path: str | Path) -> dict:
    """Read a seed file into {field: float32 array of nx_file}."""
    data = Path(path).read_bytes()
    if len(data) < 8:
        raise SeedError(f"seed file too short: {path}")
    n_fields, nx_file = struct.unpack("<ii", data[:8])
    if n_fields < 1 or nx_file < 2:
        raise SeedError(f"bad seed header ({n_fields}, {nx_file}) in {path}")
    n_load = min(n_fields, 6)
    need = 8 + 4 * n_load * nx_file
    if len(data) < need:
        raise SeedError(f"seed file {path} truncated: {len(data)} < {need} bytes")
    vals = np.frombuffer(data, dtype="<f4", count=n_load * nx_file, offset=8).reshape(n_load, nx_file)
    return {FIELD_ORDER[k]: vals[k].copy() for k in range(n_load)}


def interpolate(profile: np.ndarray, nx: int) -> np.ndarray:
    """Float32 linear interpolation of one profile to nx points (main_ym.cu:200-206)."""
    h = np.asarray(profile, dtype=np.float32)
    nf = h.shape[0]
    if nx < 2:
        raise SeedError("NX must be >= 2")
    i = np.arange(nx, dtype=np.float32)
    t = (i * np.float32(nf - 1)) / np.float32(nx - 1)
    j = np.minimum(t.astype(np.int32), nf - 2)
    frc = (t - j.astype(np.float32)).astype(np.float32)
    one = np.float32(1.0)
    out = h[j] * (one - frc) + h[j + 1] * frc
    return out.astype(np.float64)


def load_profiles(path: str | Path, nx: int) -> dict:
    """Seed file -> {field: float64 array of nx}, as uploaded by the reference."""
    return {k: interpolate(v, nx) for k, v in read_seed(path).items()}


def write_seed(path: str | Path, profiles: dict) -> None:
    """Write profiles (same length, field order by, ex, ez, az, qA, qB) in the .bin format."""
    names = [k for k in FIELD_ORDER if k in profiles]
    if names != list(FIELD_ORDER[: len(names)]):
        raise SeedError("profiles must be a prefix of (by, ex, ez, az, qA, qB)")
    nxf = len(profiles[names[0]])
    with open(path, "wb") as f:
        f.write(struct.pack("<ii", len(names), nxf))
        for k in names:
            f.write(np.asarray(profiles[k], dtype="<f4").tobytes())
