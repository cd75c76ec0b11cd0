"""The column stages at every kernel form, one step of a narrow ragged grid
(NX = 40, not a multiple of the 32-column tile) against the FP64 oracle, bit
for bit.  The z-mean removal (suppress_kz0, ymgpu2d/YM_Physics.cu:272-327):
the staged-column kernel below NZ = 128 and the coalesced residue-class
kernel from 128 to 8192 (one template per NZ; 8192 is also above the
staged kernels' shared-memory limit), each summing in the
reference's halving-tree order; the z-mean of every corrected array is then
zero to rounding.  The z-hyperdiffusion: the staged-column kernel and the
segmented one."""
from __future__ import annotations

import numpy as np
import pytest

from cases import BASE

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nz", [32, 64, 128, 256, 512, 1024, 2048, 4096, 8192])
def test_zmean_step_vs_oracle(cuda, orc, nz):
    from kh_simulations_b200._lib import Grid
    from kh_simulations_b200.config import derive, loads, step_params
    from kh_simulations_b200.run import KHRun

    cfg = loads(BASE + f"nz_override = {nz}\nnx_override = 40\nsuppress_kz0 = 1\n", f"zmean_{nz}")
    d = derive(cfg)
    run = KHRun(cfg)
    run.init()
    s0 = run.state_numpy()
    run.step(1)
    s = run.state_numpy()
    run.close()
    s_orc = orc.step(Grid(d.nx, d.nz, d.dx, d.dz), step_params(cfg, d), s0.copy(), 1)
    assert np.array_equal(s.view(np.uint64), s_orc.view(np.uint64))
    # the 15 corrected arrays (By1, Ex1, Ez1, the colour-2/3 fields but Az1, and
    # Q2, Q3 of both beams) have no kz = 0 part left
    sel = s[[6, 0, 3, 7, 8, 1, 2, 4, 5, 10, 11, 16, 17, 22, 23]]
    m = np.abs(sel.mean(axis=1)).max(axis=1)
    scale = np.abs(sel).max(axis=(1, 2)) + 1e-300
    assert (m / scale < 1e-12).all(), m / scale


@pytest.mark.parametrize("nz", [32, 64, 96, 128, 1024])
def test_hyperdiff_step_vs_oracle(cuda, orc, nz):
    """z-hyperdiffusion (ymgpu2d/YM_Physics.cu:228-259, read from the values
    before the update): the staged-column kernel at NZ = 32 and the
    segmented kernel (NZ a multiple of 32 from 64; 2-row segments at 64,
    3-row at 96), one step against the oracle bit for bit."""
    from kh_simulations_b200._lib import Grid
    from kh_simulations_b200.config import derive, loads, step_params
    from kh_simulations_b200.run import KHRun

    cfg = loads(BASE + f"nz_override = {nz}\nnx_override = 40\nhyp_diff = 5e-5\n", f"hyperdiff_{nz}")
    d = derive(cfg)
    run = KHRun(cfg)
    run.init()
    s0 = run.state_numpy()
    run.step(1)
    s = run.state_numpy()
    run.close()
    s_orc = orc.step(Grid(d.nx, d.nz, d.dx, d.dz), step_params(cfg, d), s0.copy(), 1)
    assert np.array_equal(s.view(np.uint64), s_orc.view(np.uint64))
