"""Make tests/golden/growth_fits.json: amplitude histories and the growth
rates that the reference's own fitters give on them.

Run with the reference's ymgpu2d tree at hand:

    python tests/golden/make_growth_fixtures.py <reference>/ymgpu2d

Inputs:
- the eleven runs of the reference's resolution study
  (ymgpu2d/analysis/resconv_data.json): times, |By2 + i By3| amplitudes at
  kz = 1 and the window fit stored beside them;
- seeded synthetic histories (numpy default_rng(7)): exponential growth
  with saturation and noise, of several lengths.

Also the reference's WKB growth rate (batch_analyze.py:19-41) on a grid of
(alpha, V0, kz).  Outputs for every history: the reference's fit_growth_rate and
fit_growth_rate_plateau (ymgpu2d/analysis/batch_analyze.py:44-150) and its
windowed fit (ymgpu2d/analysis/resolution_convergence.py:89-125), computed by
importing those modules.  resolution_convergence imports matplotlib, which
is absent here; a stub module stands in for it (no plotting is called).
The physics settings of the study's runs (RESOLUTION_FINDINGS.md "Fixed
physics baseline", gen_lx_resolution_campaign.py:40-54) are stored with
them, for the GPU test that reruns three of them.
"""
import json
import sys
import types
from pathlib import Path

import numpy as np

def _ref_dir() -> Path:
    """The reference's ymgpu2d tree: the first argument, else $YMKH_REFERENCE_DIR."""
    import os

    arg = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("YMKH_REFERENCE_DIR")
    if not arg:
        sys.exit(f"usage: python {Path(__file__).name} <reference ymgpu2d dir>  (or set YMKH_REFERENCE_DIR)")
    return Path(arg)


REF = _ref_dir() if __name__ == "__main__" else None
OUT = Path(__file__).resolve().parent / "growth_fits.json"


def _import_reference():
    for name in ("matplotlib", "matplotlib.pyplot"):
        mod = types.ModuleType(name)
        mod.use = lambda *a, **k: None
        sys.modules.setdefault(name, mod)
    sys.modules["matplotlib"].pyplot = sys.modules["matplotlib.pyplot"]
    sys.path.insert(0, str(REF / "analysis"))
    import batch_analyze  # noqa: E402
    import resolution_convergence  # noqa: E402
    return batch_analyze, resolution_convergence


def _synthetic(rng):
    out = []
    for n, dt, gamma, sat, noise in [(120, 1.0, 0.09, 40.0, 0.02), (400, 0.5, 0.15, 60.0, 0.05),
                                     (60, 2.0, 0.05, 1e9, 0.01), (30, 1.0, 0.2, 15.0, 0.1)]:
        t = np.arange(n) * dt
        a = 1e-8 * np.exp(gamma * t) / (1.0 + np.exp(gamma * (t - sat)))
        a = a * np.exp(noise * rng.standard_normal(n))
        out.append((f"synthetic_n{n}_g{gamma}", t, a))
    return out


def main():
    ba, rc = _import_reference()
    data = json.loads((REF / "analysis" / "resconv_data.json").read_text())
    cases = []
    series = [(k, np.array(v["times"]), np.array(v["amps"])) for k, v in data.items()]
    series += _synthetic(np.random.default_rng(7))
    for name, t, a in series:
        g, t0, t1, r2 = ba.fit_growth_rate(t, a, t_min=10.0)
        gw, tw0, tw1, rw2 = rc.fit_growth_rate(t, a, t_min=10.0)
        pl = ba.fit_growth_rate_plateau(t, a)
        case = {"name": name, "times": t.tolist(), "amps": a.tolist(),
                "fit": [float(g), float(t0), float(t1), float(r2)],
                "window_fit": [float(gw), float(tw0), float(tw1), float(rw2)],
                "plateau": {k: (float(v) if not isinstance(v, bool) else v) for k, v in pl.items()}}
        if name in data:
            v = data[name]
            case["stored_window_fit"] = [v["gamma"], v["gamma_fit_t0"], v["gamma_fit_t1"], v["gamma_r2"]]
            case["grid"] = {"nx": v["nx"], "nz": v["nz"], "dt": v["dt"]}
        cases.append(case)
    physics = {"k_mode": 1, "alpha_YM": 1.0, "V0": 0.05, "perturb_amp": 0.001, "run_mode": 6,
               "xi_sponge": 10.0, "sigma_sponge": 5.0, "suppress_kz0": 1, "hyp_diff": "5e-5",
               "kz_suppress_max": 0, "eps_override": 0.15, "kz_suppress_hi": 14, "target_tu": 25.0}
    runs = {"res_baseline": {"nz_override": 256, "nx_override": 768, "courant_override": 0.01},
            "res_nz128": {"nz_override": 128, "nx_override": 384, "courant_override": 0.01},
            "res_c0.04": {"nz_override": 256, "nx_override": 768, "courant_override": 0.04}}
    wkb = [[a, v, k, float(ba.wkb_exact_gamma(a, v, k))]
           for a in (0.0, 0.1, 0.5, 1.0, 2.5, 6.0) for v in (0.01, 0.05, 0.2) for k in (0.125, 0.5, 1.0, 3.0, 7.0)]
    OUT.write_text(json.dumps({"source": "ymgpu2d/analysis/resconv_data.json + seeded synthetic histories",
                               "t_min": 10.0, "physics": physics, "runs": runs, "cases": cases,
                               "wkb_exact_gamma": wkb}, indent=1) + "\n")
    print(f"wrote {OUT} ({len(cases)} histories)")


if __name__ == "__main__":
    main()
