"""The CUDA path against the reference's own outputs stored in
tests/golden/ (made by tests/golden/make_golden.py from the reference's
kernels, compiled from its unmodified sources with -fmad=false, on a B200).
Needs no reference build at run time.

For every stored case: the initial state of ymkh_init equals the
reference's bit for bit; from it, the state after the stored steps equals
the reference's bit for bit without a band filter, and within the band
filter's 1e-12 (per field, over the largest norm in its group) with one;
the energy is the reference's within 1e-13 (compensated sum against its
sequential host sum).
"""
from pathlib import Path

import numpy as np
import pytest

from cases import BITWISE, GOLDEN, golden_config
from test_gpu_parity import FILTER_TOL, rel_l2

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
    if name in BITWISE:
        assert np.array_equal(s1, ref), f"max |diff| {np.abs(s1 - ref).max()}"
    else:
        assert rel_l2(s1, ref).max() < FILTER_TOL, rel_l2(s1, ref)
    e = run.energy()
    assert abs(e - float(z["e1"])) <= 1e-13 * abs(float(z["e1"]))
    run.close()
