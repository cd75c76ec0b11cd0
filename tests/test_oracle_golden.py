"""Pins the FP64 CPU oracle to the reference itself: golden vectors made by
tests/golden/make_golden.py from the reference's own kernels (compiled from
its unmodified sources, -fmad=false) on a B200.  The oracle, started from the
reference's initial state and given the GPU's FP32 twiddle table, must
reproduce the reference's state after the stored steps bit for bit, and the
reference's energy (per-cell formula and sequential sum) exactly."""
from pathlib import Path

import numpy as np
import pytest

from cases import GOLDEN, golden_config

GOLD = Path(__file__).resolve().parent / "golden"


def _load(name):
    f = GOLD / f"{name}.npz"
    if not f.exists():
        pytest.fail(f"missing golden fixture {f}")
    return np.load(f)


@pytest.mark.parametrize("name", GOLDEN)
def test_oracle_reproduces_reference(orc, name):
    from kh_simulations_b200._lib import Grid
    from kh_simulations_b200.config import derive, loads, step_params

    z = _load(name)
    cfg = loads(str(z["ini"]), name)
    assert cfg == golden_config(name)
    d = derive(cfg)
    g = Grid(d.nx, d.nz, d.dx, d.dz)
    p = step_params(cfg, d)
    tw = np.load(GOLD / "twiddles_nz32.npz")
    s = np.ascontiguousarray(z["init"])
    assert orc.energy(g, s) == float(z["e0"])
    orc.step(g, p, s, int(z["steps"]), twiddles=(tw["cos"], tw["sin"]))
    ref = z["final"]
    assert np.array_equal(s, ref), f"max |diff| {np.abs(s - ref).max()}"
    assert orc.energy(g, s) == float(z["e1"])


def test_host_twiddles_close_to_gpu_table(orc):
    """The C library's cosf/sinf agree with the GPU's to a couple of ulps;
    the GPU table is the one parity uses."""
    tw = np.load(GOLD / "twiddles_nz32.npz")
    c, s = orc.twiddles(32, 0, tw["cos"].shape[0] - 1)
    assert np.max(np.abs(c - tw["cos"])) <= 2.5e-7
    assert np.max(np.abs(s - tw["sin"])) <= 2.5e-7


def test_oracle_uniform_state(orc):
    """A uniform fluid at rest with empty fields is a fixed point of the step
    without band filters.  With a band filter it is not: the reference's FP32
    twiddles are not orthogonal to a constant, so n picks up a leak of order
    the FP32 phase error (a reference property the oracle reproduces)."""
    from kh_simulations_b200._lib import Grid
    from kh_simulations_b200.config import derive, loads, step_params

    def run(text):
        cfg = loads(text)
        d = derive(cfg)
        s = np.zeros((24, d.nz, d.nx))
        s[12] = s[18] = 1.0
        orc.step(Grid(d.nx, d.nz, d.dx, d.dz), step_params(cfg, d), s, 3)
        return s

    s = run("nz_override = 32\nnx_override = 16\nsuppress_kz0 = 1\nhyp_diff = 1e-4\n")
    assert np.all(s[12] == 1.0) and np.all(s[18] == 1.0)
    assert np.count_nonzero(np.delete(s, [12, 18], axis=0)) == 0
    s = run("nz_override = 32\nnx_override = 16\nkz_keep_max = 10\n")
    leak = np.abs(s[12] - 1.0).max()
    assert 0 < leak < 1e-5
    assert np.count_nonzero(np.delete(s, [12, 18], axis=0)) == 0
