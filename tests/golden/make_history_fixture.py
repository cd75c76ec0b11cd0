"""Make tests/golden/history_config0.npz: the energy every 10 steps and the
k = 1 mode amplitude every 100 steps of the reference's own kernels
(oracle/_ref, -fmad=false) on the config-0 run (NZ 256 x NX 512, keep
|k| <= 85) over 10^4 steps or until its halt rule
(ymgpu2d/main_ym.cu:249, 467-474).  Needs a GPU and the reference harness
built (make -C oracle ref).  Usage:

    python tests/golden/make_history_fixture.py OUTDIR
"""
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))

from cases import BASE  # noqa: E402
from kh_simulations_b200._lib import Grid  # noqa: E402
from kh_simulations_b200.config import derive, loads, step_params  # noqa: E402
from kh_simulations_b200.run import init_params  # noqa: E402
from oracle import RefHarness  # noqa: E402

INI = BASE + "nz_override = 256\nnx_override = 512\nkz_keep_max = 85\n"


def main(out: Path) -> None:
    out.mkdir(parents=True, exist_ok=True)
    cfg = loads(INI, "config0")
    d = derive(cfg)
    ref = RefHarness(parity=True)
    ref.create(Grid(d.nx, d.nz, d.dx, d.dz), step_params(cfg, d))
    ip, _k = init_params(cfg, d)
    ref.init(ip)
    e0 = ref.energy()
    energies, amps = [], []
    halted_at = -1
    for i in range(1, 1001):
        ref.step(10)
        e = ref.energy()
        if not np.isfinite(e) or e / e0 > d.energy_thresh:
            halted_at = 10 * i
            break
        energies.append(e)
        if i % 10 == 0:
            s = ref.get_state()
            amps.append(np.abs(np.fft.fft(s[10] + 1j * s[11], axis=0)[1]).mean() / d.nz)
    ref.destroy()
    np.savez_compressed(out / "history_config0.npz", ini=INI, e0=e0, energy_every_10=np.array(energies),
                        mode1_every_100=np.array(amps), halted_at=halted_at)
    print(f"{len(energies)} energy checks, {len(amps)} amplitudes, halted at {halted_at}")


if __name__ == "__main__":
    main(Path(sys.argv[1]))
