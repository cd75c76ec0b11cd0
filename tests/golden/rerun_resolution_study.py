"""Rerun runs of the reference's resolution study with the reference's own
kernels (oracle/_ref, both builds) and with this build, and print how far
each amplitude history lies from the one the reference recorded
(tests/golden/growth_fits.json, from ymgpu2d/analysis/resconv_data.json).

Needs a GPU and oracle/_ref built (make -C oracle ref).  Usage:

    python tests/golden/rerun_resolution_study.py res_nz128 res_baseline

The spread between the reference's two builds (FMA contraction off / on)
shows how sensitive a run is to rounding; tests/test_gpu_physics.py sets its
tolerances from what this printed on a B200.
"""
import json
import math
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from kh_simulations_b200 import growth  # noqa: E402
from kh_simulations_b200._lib import Grid  # noqa: E402
from kh_simulations_b200.config import derive, loads, step_params  # noqa: E402
from kh_simulations_b200.run import KHRun, init_params  # noqa: E402
from oracle import RefHarness  # noqa: E402
from oracle import diagnostics as od  # noqa: E402

FIX = json.loads((Path(__file__).parent / "growth_fits.json").read_text())


def ini(name):
    k = dict(FIX["physics"])
    k.update(FIX["runs"][name])
    return "".join(f"{a} = {b}\n" for a, b in k.items())


def main(names):
    for name in names:
        case = next(c for c in FIX["cases"] if c["name"] == name)
        cfg = loads(ini(name), name)
        d = derive(cfg)
        w = growth.xi_weight(d.nx, d.dx, eps=0.15, lx=6 * math.pi)
        rec = np.array(case["amps"])
        hist = {}
        for parity in (True, False):
            h = RefHarness(parity=parity)
            h.create(Grid(d.nx, d.nz, d.dx, d.dz), step_params(cfg, d))
            ip, _keep = init_params(cfg, d)
            h.init(ip)
            amps, t0 = [], time.time()
            for k in range(len(rec)):
                if k:
                    h.step(d.export_stride)
                st = h.get_state()
                amps.append(od.circ_amp(st[od.IDX["By2"]], st[od.IDX["By3"]], 1, w)[0])
            h.destroy()
            hist["reference -fmad=false" if parity else "reference stock"] = np.array(amps)
            print(f"{name}: reference {'parity' if parity else 'stock'} build, {time.time() - t0:.0f} s", flush=True)
        run = KHRun(cfg)
        run.init()
        ours = []
        run.run(on_export=lambda r, s: ours.append(r.circ_amp("By", k=1, weight=w)[0]))
        run.close()
        hist["this build"] = np.array(ours)
        t = np.arange(len(rec)) * d.export_stride * d.dt
        print(f"{name}: |amp / recorded - 1| at t = " + " ".join(f"{x:5.1f}" for x in t[1::3]))
        for k, a in hist.items():
            g = growth.fit_growth_rate_window(t, a, t_min=FIX["t_min"])[0]
            print(f"  {k:22s} " + " ".join(f"{x:.1e}" for x in np.abs(a[1:] / rec[1:] - 1)[::3])
                  + f"   gamma {g:.7f} (recorded {case['stored_window_fit'][0]:.7f})")


if __name__ == "__main__":
    main(sys.argv[1:] or sorted(FIX["runs"]))
