"""Physics pin: runs of the reference's resolution study, rerun through
KHRun and compared with the amplitude histories the reference recorded.

tests/golden/growth_fits.json (made by tests/golden/make_growth_fixtures.py
from ymgpu2d/analysis/resconv_data.json) holds, for each run, |By2 + i By3|
at kz = 1, sech-weighted over x, every export stride (1 TU) for 25 TU, as
the reference's analysis computed it from its 6-digit CSV snapshots, and
the growth rate it fitted (ymgpu2d/analysis/resolution_convergence.py).
The settings are the study's fixed physics baseline (kz = 1, alpha = 1,
V0 = 0.05, EPS = 0.15, mode 6, sponge 10/5, hyperdiffusion 5e-5, z-mean
removal, modes 2..14 subtracted) with each run's grid and Courant number.

The whole step runs for 25,000 to 100,000 steps here: every stage,
including the sponge, z-mean, band filter and hyperdiffusion, against an
independent record of the reference's own trajectory.  The record carries
6 digits (CSV snapshots) and came from the reference's stock build on
other GPUs.  Rerun on a B200 (tests/golden/rerun_resolution_study.py), the
histories of the reference's own kernels and of this build lie from it:

  run           t <= 19      t = 25     gamma vs recorded
  res_baseline  all < 1e-6   < 3.1e-5   < 1.1e-5 (all three)
  res_c0.04     this build 4.2e-7 over the whole run, gamma equal to 6 digits
  res_nz128     all < 3e-6   stock 2.1e-4, -fmad=false 1.3e-3, this build
                1.5e-3; gamma: stock 4.7e-4, -fmad=false 1.3e-3, this
                build 2.0e-3

The coarse res_nz128 run is sensitive to rounding after t ~ 20: the
reference's two builds, which differ only in FMA contraction, part by
1.1e-3 there.  This build also differs from the reference in the band
filter's summation order (1e-12 relative per step) and reads a copy where
the reference's hyperdiffusion races, so it lies a little further out.
Tolerances: amplitudes within AMP_RTOL up to t = 19 in every run and over
the whole run where the reference is not sensitive; within LATE_RTOL after
t = 19 in res_nz128; growth rates within GAMMA_RTOL, LATE_RTOL in
res_nz128.
"""
import json
import math
from pathlib import Path

import numpy as np
import pytest

from kh_simulations_b200 import growth
from kh_simulations_b200.config import loads
from kh_simulations_b200.run import KHRun

pytestmark = pytest.mark.gpu

FIX = json.loads((Path(__file__).parent / "golden" / "growth_fits.json").read_text())
AMP_RTOL = 1e-4
GAMMA_RTOL = 1e-4
LATE_RTOL = 5e-3
SENSITIVE = {"res_nz128"}  # runs whose history parts with rounding after t = 19


def _ini(run_name: str) -> str:
    keys = dict(FIX["physics"])
    keys.update(FIX["runs"][run_name])
    return "".join(f"{k} = {v}\n" for k, v in keys.items())


@pytest.mark.parametrize("run_name", sorted(FIX["runs"]))
def test_resolution_study_history(run_name):
    case = next(c for c in FIX["cases"] if c["name"] == run_name)
    run = KHRun(loads(_ini(run_name), run_name))
    d = run.d
    assert (d.nx, d.nz) == (case["grid"]["nx"], case["grid"]["nz"])
    assert d.dt == pytest.approx(case["grid"]["dt"], rel=1e-7)  # theirs is inferred from 9-digit CSV times
    w = growth.xi_weight(d.nx, d.dx, eps=0.15, lx=6.0 * math.pi)
    rec = []
    run.init()
    run.run(on_export=lambda r, s: rec.append((s, r.circ_amp("By", k=1, weight=w)[0])))
    assert not run.halted, run.halt_reason
    steps = np.array([s for s, _ in rec])
    amps = np.array([a for _, a in rec])
    ref_t, ref_a = np.array(case["times"]), np.array(case["amps"])
    assert len(steps) == len(ref_t)
    assert np.array_equal(steps, np.rint(ref_t / case["grid"]["dt"]).astype(int))
    assert amps[0] == 0.0 and ref_a[0] == 0.0
    rel = np.abs(amps[1:] / ref_a[1:] - 1.0)
    t = ref_t[1:]
    print(f"{run_name}: amplitude rel diff max {rel[t <= 19.5].max():.3e} up to t=19, {rel.max():.3e} overall")
    assert rel[t <= 19.5].max() < AMP_RTOL
    assert rel.max() < (LATE_RTOL if run_name in SENSITIVE else AMP_RTOL)
    g, t0, t1, r2 = growth.fit_growth_rate_window(steps * d.dt, amps, t_min=FIX["t_min"])
    ref_g = case["stored_window_fit"][0]
    print(f"{run_name}: gamma {g:.7f} (recorded {ref_g:.7f}), window [{t0:.2f}, {t1:.2f}], R2 {r2:.5f}")
    assert g == pytest.approx(ref_g, rel=LATE_RTOL if run_name in SENSITIVE else GAMMA_RTOL)
    run.close()
