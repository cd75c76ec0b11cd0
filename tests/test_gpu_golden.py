"""The CUDA path against the reference's own outputs stored in
tests/golden/ (made by tests/golden/make_golden.py from the reference's
kernels, compiled from its unmodified sources with -fmad=false, on a B200).
Needs no reference build at run time.

For every stored case: the initial state of ymkh_init equals the
reference's bit for bit; from it, the state after the stored steps equals
the reference's bit for bit, with and without a band filter (the FP64
filter sums in the reference's warp-tree order);
the energy is the reference's within 1e-13 (compensated sum against its
sequential host sum).
"""
from pathlib import Path

import numpy as np
import pytest

from cases import GOLDEN, golden_config

pytestmark = pytest.mark.gpu

GOLD = Path(__file__).resolve().parent / "golden"


@pytest.mark.parametrize("name", GOLDEN)
def test_cuda_path_reproduces_reference_fixture(cuda, name):
    from kh_simulations_b200.run import KHRun

    z = np.load(GOLD / f"{name}.npz")
    run = KHRun(golden_config(name))
    run.init()
    s0 = run.state_numpy()
    assert np.array_equal(s0.view(np.uint64), z["init"].view(np.uint64)), "initial state"
    run.step(int(z["steps"]))
    s1 = run.state_numpy()
    ref = z["final"]
    assert np.array_equal(s1, ref), f"max |diff| {np.abs(s1 - ref).max()}"
    e = run.energy()
    assert abs(e - float(z["e1"])) <= 1e-13 * abs(float(z["e1"]))
    run.close()


def test_config0_history_vs_reference_fixture(cuda):
    """The config-0 run (NZ 256 x NX 512, keep |k| <= 85) against the
    reference's stored history (tests/golden/make_history_fixture.py): the
    energy every 10 steps within 1e-9, the k = 1 amplitude every 100 steps
    within 1e-9, and the halt rule stopping both at the same check."""
    from kh_simulations_b200.config import loads
    from kh_simulations_b200.run import KHRun

    z = np.load(GOLD / "history_config0.npz")
    run = KHRun(loads(str(z["ini"]), "config0"))
    run.init()
    e0 = run.energy()
    # compensated sum against the reference's sequential host sum over
    # 131,072 cells: the latter's rounding is ~1e-13 relative here
    assert abs(e0 - float(z["e0"])) <= 1e-12 * abs(float(z["e0"]))
    ref_e, ref_a = z["energy_every_10"], z["mode1_every_100"]
    energies, amps, halted_at = [], [], -1
    for i in range(1, 1001):
        run.step(10)
        e = run.energy()
        if not np.isfinite(e) or e / e0 > run.d.energy_thresh:
            halted_at = 10 * i
            break
        energies.append(e)
        if i % 10 == 0:
            amps.append(run.mode_amp(1)[0])
    assert halted_at == int(z["halted_at"])
    assert len(energies) == len(ref_e) and len(ref_e) >= 100
    dev = np.abs(np.array(energies) - ref_e) / np.abs(ref_e)
    assert dev.max() < 1e-9, (dev.max(), int(dev.argmax()))
    assert np.all(np.abs(np.array(amps) - ref_a) <= 1e-9 * np.abs(ref_a))
    run.close()
