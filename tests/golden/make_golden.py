"""Generates the golden vectors of tests/golden/ from the REFERENCE ITSELF.

Runs on a machine with a GPU and the reference harness built
(``make -C oracle ref``: the reference's own kernels from its unmodified
sources, -fmad=false).  For every case in tests/cases.py GOLDEN it stores the
reference's initial state, its state after GOLDEN_STEPS steps and the
reference's energy of both (ymgpu2d/YM_Energy.cu host sum), plus the FP32
filter twiddle table evaluated on the GPU.  Usage:

    python tests/golden/make_golden.py OUTDIR
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))

from cases import CASES, GOLDEN, GOLDEN_STEPS, golden_config  # noqa: E402
from kh_simulations_b200 import _lib  # noqa: E402
from kh_simulations_b200._lib import Grid  # noqa: E402
from kh_simulations_b200.config import derive, step_params  # noqa: E402
from kh_simulations_b200.run import init_params  # noqa: E402
from oracle import RefHarness  # noqa: E402


def main(out: Path) -> None:
    out.mkdir(parents=True, exist_ok=True)
    ref = RefHarness(parity=True)
    for name in GOLDEN:
        cfg = golden_config(name)
        d = derive(cfg)
        p = step_params(cfg, d)
        g = Grid(d.nx, d.nz, d.dx, d.dz)
        ip, _keep = init_params(cfg, d)
        ref.create(g, p)
        ref.init(ip)
        s0 = ref.get_state()
        e0 = ref.energy()
        ref.step(GOLDEN_STEPS)
        s1 = ref.get_state()
        e1 = ref.energy()
        np.savez_compressed(out / f"{name}.npz", init=s0, final=s1, e0=e0, e1=e1, steps=GOLDEN_STEPS,
                            ini=CASES[name].replace("nx_override = 48", "nx_override = 32"))
        print(name, d.nx, d.nz, e0, e1, flush=True)
    ref.destroy()
    # FP32 filter twiddles on the GPU (the expression of YM_Physics.cu:387-388)
    import ctypes as C
    lib = _lib.load()
    nz, mhi = 32, 16
    c = np.empty((mhi + 1) * nz, np.float32)
    s = np.empty((mhi + 1) * nz, np.float32)
    _lib.check(lib.ymkh_twiddles(nz, 0, mhi, c.ctypes.data_as(C.c_void_p), s.ctypes.data_as(C.c_void_p)),
               "ymkh_twiddles")
    np.savez_compressed(out / "twiddles_nz32.npz", cos=c.reshape(mhi + 1, nz), sin=s.reshape(mhi + 1, nz))


if __name__ == "__main__":
    main(Path(sys.argv[1] if len(sys.argv) > 1 else ROOT / "tests" / "golden"))
