"""Growth-rate fitters against the reference's own fitters (CPU).

tests/golden/growth_fits.json holds amplitude histories (the reference's
resolution-study runs and seeded synthetic ones) with what
ymgpu2d/analysis/batch_analyze.py:44-150 and
ymgpu2d/analysis/resolution_convergence.py:89-125 return on them.  The
windows chosen must be the same and the rates equal to 1e-12.
"""
import json
import math
from pathlib import Path

import numpy as np
import pytest

from kh_simulations_b200 import growth

FIX = json.loads((Path(__file__).parent / "golden" / "growth_fits.json").read_text())
CASES = FIX["cases"]


def _close(a, b, rtol=1e-12):
    if math.isnan(b):
        return math.isnan(a)
    return abs(a - b) <= rtol * max(abs(b), 1e-300)


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_best_window_fit(case):
    g, t0, t1, r2 = growth.fit_growth_rate(case["times"], case["amps"], t_min=FIX["t_min"])
    rg, rt0, rt1, rr2 = case["fit"]
    assert (t0, t1) == (rt0, rt1)
    assert _close(g, rg) and _close(r2, rr2)


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_fixed_window_fit(case):
    out = growth.fit_growth_rate_window(case["times"], case["amps"], t_min=FIX["t_min"])
    ref = case["window_fit"]
    assert (out[1], out[2]) == (ref[1], ref[2])
    assert _close(out[0], ref[0]) and _close(out[3], ref[3])
    if "stored_window_fit" in case:  # what the reference stored beside its data
        assert _close(out[0], case["stored_window_fit"][0], 1e-12)


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_plateau_fit(case):
    out = growth.fit_growth_rate_plateau(case["times"], case["amps"])
    ref = case["plateau"]
    assert out["has_plateau"] == ref["has_plateau"]
    for k in ("gamma", "t0", "t1", "duration"):
        assert _close(out[k], ref[k]), k


def test_fits_recover_a_clean_exponential():
    t = np.arange(0.0, 60.0, 0.5)
    a = 3e-9 * np.exp(0.0875 * t)
    assert growth.fit_growth_rate(t, a)[0] == pytest.approx(0.0875, rel=1e-12)
    assert growth.fit_growth_rate_window(t, a)[0] == pytest.approx(0.0875, rel=1e-12)
    p = growth.fit_growth_rate_plateau(t, a)
    assert p["has_plateau"] and p["gamma"] == pytest.approx(0.0875, rel=1e-12)


def test_short_and_decaying_histories():
    assert growth.fit_growth_rate([0, 1, 2], [1, 2, 4])[0] == 0.0
    assert math.isnan(growth.fit_growth_rate_window([0, 1, 2, 3], [1, 2, 4, 8])[0])
    t = np.arange(20.0)
    g, t0, t1, r2 = growth.fit_growth_rate(t, np.exp(-0.1 * t))
    assert g == 0.0 and math.isnan(t0) and r2 == -1e9
    assert not growth.fit_growth_rate_plateau(t, np.exp(-0.1 * t))["has_plateau"]


def test_xi_weight_is_a_normalised_sech():
    w = growth.xi_weight(768, 6 * math.pi / 768, eps=0.15)
    assert w.sum() == pytest.approx(1.0, abs=1e-15)
    assert int(np.argmax(w)) == 384


def test_wkb_exact_gamma_matches_the_reference():
    for alpha, v0, kz, ref in FIX["wkb_exact_gamma"]:
        assert growth.wkb_exact_gamma(alpha, v0, kz) == pytest.approx(ref, rel=1e-12, abs=1e-300), (alpha, v0, kz)
