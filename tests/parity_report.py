"""Per-field relative L2 errors of a state against a reference state, in the
two normalisations the parity tests use, and an optional JSON-lines report.

raw:   each field's L2 error over that field's own L2 norm (the bar as the
       single-run target states it, 1e-12 per field);
group: each field's L2 error over the largest norm in its physical group
       (E, By, Az, n, p, Q of each beam).  Some fields are cancellation
       residues: with symmetric counter-streaming beams Ex1 and Ez1 are sums
       of nearly cancelling beam currents, ~1e-12 beside Ex2 ~ 1e-5, so
       their own norm is no scale for a rounding difference of the band
       filter's summation order.

Set YMKH_PARITY_REPORT to a file path to have every call of `record`
append one JSON line (case, step count, both vectors, fields over 1e-12).
"""
from __future__ import annotations

import json
import os

import numpy as np

NAMES = ("Ex1", "Ex2", "Ex3", "Ez1", "Ez2", "Ez3", "By1", "By2", "By3", "Az1", "Az2", "Az3",
         "nA", "pxA", "pzA", "Q1A", "Q2A", "Q3A", "nB", "pxB", "pzB", "Q1B", "Q2B", "Q3B")
GROUPS = [range(0, 6), range(6, 9), range(9, 12), [12], [13, 14], range(15, 18), [18], [19, 20], range(21, 24)]


def _norms(a, b):
    a = np.asarray(a).reshape(24, -1)
    b = np.asarray(b).reshape(24, -1)
    num = np.sqrt(np.sum((a - b) ** 2, axis=1))
    nrm = np.sqrt(np.sum(b ** 2, axis=1))
    return num, nrm


def _div(num, den):
    return np.where(den > 0, num / np.where(den > 0, den, 1), num)


def rel_l2_group(a, b) -> np.ndarray:
    num, nrm = _norms(a, b)
    den = np.empty_like(nrm)
    for g in GROUPS:
        g = list(g)
        den[g] = nrm[g].max()
    return _div(num, den)


def rel_l2_raw(a, b) -> np.ndarray:
    num, nrm = _norms(a, b)
    return _div(num, nrm)


def norms(b) -> np.ndarray:
    return np.sqrt(np.sum(np.asarray(b).reshape(24, -1) ** 2, axis=1))


def record(case: str, steps: int, a, b, note: str = "") -> dict:
    """Both normalisations of a against b; appended to $YMKH_PARITY_REPORT."""
    g, r = rel_l2_group(a, b), rel_l2_raw(a, b)
    nb = norms(b)
    rep = {"case": case, "steps": steps, "note": note,
           "max_group": float(g.max()), "max_raw": float(r.max()),
           "raw_over_1e-12": {NAMES[i]: {"raw": float(r[i]), "group": float(g[i]), "norm": float(nb[i])}
                              for i in range(24) if r[i] > 1e-12},
           "raw": {NAMES[i]: float(r[i]) for i in range(24)},
           "group": {NAMES[i]: float(g[i]) for i in range(24)}}
    path = os.environ.get("YMKH_PARITY_REPORT")
    if path:
        with open(path, "a") as f:
            f.write(json.dumps(rep) + "\n")
    return rep
