"""Growth-rate extraction from a mode-amplitude history.

The reference fits the linear growth rate gamma of the Kelvin–Helmholtz
mode offline, from CSV snapshots.  Here the amplitudes come from the device
(``KHRun.circ_amp`` at the export stride) and these functions fit them on
the host.  Three fitters are kept, each giving what the reference's gives
on the same history:

- ``fit_growth_rate``: best-R^2 straight line of ln(amp) over every window
  of at least ``min_win_frac`` of the samples
  (ymgpu2d/analysis/batch_analyze.py:44-70).
- ``fit_growth_rate_window``: best-R^2 fixed-length window over a 7-sample
  moving mean of ln(amp) (ymgpu2d/analysis/resolution_convergence.py:89-125).
- ``fit_growth_rate_plateau``: the longest run of samples whose local slope
  stays flat, then one fit over it (ymgpu2d/analysis/batch_analyze.py:73-150).

The least-squares lines are computed from window sums of data centred on
their global means (one pass for all windows of a length), not one
polynomial fit per window.
"""
from __future__ import annotations

import math

import numpy as np

_TINY = 1e-30


def xi_weight(nx: int, dx: float, eps: float = 0.15, lx: float = 6.0 * math.pi) -> np.ndarray:
    """sech((x - lx/2)/eps) over x = i*dx, normalised to sum 1: the shear-layer
    weight of the x-average (ymgpu2d/analysis/resolution_convergence.py:77-80)."""
    x = np.arange(nx) * dx
    w = 1.0 / np.cosh((x - lx / 2.0) / eps)
    return w / w.sum()


def _line_fits(t: np.ndarray, a: np.ndarray, length: int):
    """Slope and R^2 of the least-squares line through every window
    t[i:i+length], a[i:i+length]; R^2 = 1 - ss_res / (ss_tot + 1e-30)."""
    t = t - t.mean()
    a = a - a.mean()

    def wsum(v):
        c = np.concatenate(([0.0], np.cumsum(v)))
        return c[length:] - c[:-length]

    n = float(length)
    st, sa = wsum(t), wsum(a)
    stt = wsum(t * t) - st * st / n
    sta = wsum(t * a) - st * sa / n
    saa = wsum(a * a) - sa * sa / n
    slope = sta / stt
    ss_res = np.maximum(saa - slope * sta, 0.0)
    r2 = 1.0 - ss_res / (saa + _TINY)
    return slope, r2


def fit_growth_rate(times, amps, t_min=None, t_max=None, min_win_frac: float = 0.15):
    """(gamma, t0, t1, r2) of the best-R^2 window of ln(amp) with a slope of
    at least 1e-6, over every window [i, j) of at least
    max(4, int(n * min_win_frac)) samples.  Ties keep the window met first
    in the order (i ascending, then j ascending).  (0.0, nan, nan, 0.0) when
    fewer than 4 samples lie in [t_min, t_max]."""
    times = np.asarray(times, dtype=np.float64)
    log_a = np.log(np.clip(np.asarray(amps, dtype=np.float64), _TINY, None))
    m = np.ones(len(times), dtype=bool)
    if t_min is not None:
        m &= times >= t_min
    if t_max is not None:
        m &= times <= t_max
    tw, aw = times[m], log_a[m]
    n = len(tw)
    if n < 4:
        return 0.0, math.nan, math.nan, 0.0
    min_win = max(4, int(n * min_win_frac))
    best_r2, best, best_key = -1e9, (0.0, math.nan, math.nan), None
    for length in range(min_win, n + 1):
        slope, r2 = _line_fits(tw, aw, length)
        ok = slope >= 1e-6
        if not ok.any():
            continue
        r2m = np.where(ok, r2, -np.inf)
        i = int(np.argmax(r2m))
        if r2m[i] > best_r2 or (r2m[i] == best_r2 and best_key is not None and i < best_key[0]):
            best_r2, best, best_key = float(r2m[i]), (float(slope[i]), float(tw[i]), float(tw[i + length - 1])), (i, length)
    return best[0], best[1], best[2], best_r2


def _moving_mean(v: np.ndarray, half: int = 3) -> np.ndarray:
    n = len(v)
    c = np.concatenate(([0.0], np.cumsum(v)))
    i = np.arange(n)
    lo, hi = np.maximum(0, i - half), np.minimum(n, i + half + 1)
    return (c[hi] - c[lo]) / (hi - lo)


def fit_growth_rate_window(times, amps, t_min=None, t_max=None, min_win_frac: float = 0.3):
    """(gamma, t0, t1, r2) of the best-R^2 window of fixed length
    max(5, int(n * min_win_frac)) over the 7-sample moving mean of
    ln(amp + 1e-30), for samples in [t_min, t_max] with amp > 1e-30.
    Windows start at 0 .. max(1, n - win) - 1, so the last full window is
    not tried, as in the reference.  NaNs when fewer than 5 samples."""
    times = np.asarray(times, dtype=np.float64)
    amps = np.asarray(amps, dtype=np.float64)
    m = np.ones(len(times), dtype=bool)
    if t_min is not None:
        m &= times >= t_min
    if t_max is not None:
        m &= times <= t_max
    m &= amps > _TINY
    if m.sum() < 5:
        return math.nan, math.nan, math.nan, math.nan
    tw = times[m]
    env = _moving_mean(np.log(amps[m] + _TINY))
    n = len(tw)
    win = max(5, int(n * min_win_frac))
    starts = max(1, n - win)
    slope, r2 = _line_fits(tw, env, win)
    slope, r2 = slope[:starts], r2[:starts]
    ok = slope >= 1e-6
    if not ok.any():
        return math.nan, math.nan, math.nan, -math.inf
    r2m = np.where(ok, r2, -np.inf)
    i = int(np.argmax(r2m))
    return float(slope[i]), float(tw[i]), float(tw[i + win - 1]), float(r2m[i])


def _local_slopes(times: np.ndarray, log_a: np.ndarray, win_tu: float):
    """Slope of ln(amp) over [t_i - win_tu/2, t_i + win_tu/2] at each sample
    with at least 4 samples in that span (batch_analyze.py:73-87)."""
    half = win_tu / 2.0
    tc, sl = [], []
    for i in range(len(times)):
        m = (times >= times[i] - half) & (times <= times[i] + half)
        if m.sum() < 4:
            continue
        t, a = times[m] - times[m].mean(), log_a[m] - log_a[m].mean()
        tc.append(times[i])
        sl.append(float(np.dot(t, a) / np.dot(t, t)))
    return np.array(tc), np.array(sl)


def fit_growth_rate_plateau(times, amps, win_tu: float = 8.0, min_plateau_tu: float = 10.0,
                            flat_tol: float = 0.06) -> dict:
    """Growth rate over the longest plateau of the local slope.

    A plateau grows sample by sample from a positive local slope while the
    peak-to-peak spread of its slopes stays within ``flat_tol`` of their
    median; the longest one spanning at least ``min_plateau_tu`` is fitted
    with one line.  Returns gamma, t0, t1, duration, has_plateau."""
    times = np.asarray(times, dtype=np.float64)
    log_a = np.log(np.clip(np.asarray(amps, dtype=np.float64), _TINY, None))
    empty = {"gamma": math.nan, "t0": math.nan, "t1": math.nan, "duration": math.nan, "has_plateau": False}
    if len(times) < 8:
        return empty
    tc, sl = _local_slopes(times, log_a, win_tu)
    if len(tc) < 4:
        return empty
    pos = sl > 1e-6
    n = len(tc)
    best = None
    i = 0
    while i < n:
        if not pos[i]:
            i += 1
            continue
        lo = hi = i  # the run is tc[lo..hi]
        j = i + 1
        while j < n and pos[j]:
            vals = sl[lo:j + 1]
            med = float(np.median(vals))
            if (vals.max() - vals.min()) / med <= flat_tol:
                hi = j
                j += 1
            else:
                break
        dur = tc[hi] - tc[lo]
        if dur >= min_plateau_tu and (best is None or dur > best[2]):
            best = (lo, hi, dur)
        i = hi + 1 if hi > lo else i + 1
    if best is None:
        return empty
    t0, t1 = tc[best[0]], tc[best[1]]
    m = (times >= t0) & (times <= t1)
    t, a = times[m] - times[m].mean(), log_a[m] - log_a[m].mean()
    return {"gamma": float(np.dot(t, a) / np.dot(t, t)), "t0": float(t0), "t1": float(t1),
            "duration": float(best[2]), "has_plateau": True}


def wkb_exact_gamma(alpha: float, V0: float, kz: float) -> float:
    """Largest Im(omega) over the roots of the harmonic-core WKB quartic
    omega^4 - kz^2 omega^2 - C omega - alpha^2 V0 kz = 0 with
    C = sqrt(alpha^3 / 2) V0 (the fundamental mode), 0.0 when no root grows
    (ymgpu2d/analysis/batch_analyze.py:19-41)."""
    c = math.sqrt(alpha ** 3 / 2.0) * V0
    roots = np.roots([1.0, 0.0, -kz ** 2, -c, -alpha ** 2 * V0 * kz])
    growing = roots[roots.imag > 1e-8]
    return float(np.max(growing.imag)) if len(growing) else 0.0
