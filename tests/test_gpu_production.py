"""Parity at the sizes the benchmarks run, against the reference's own kernels.

The small-grid cases (tests/cases.py, 32 x 48) pin every stage of the step.
These cases pin the launch shapes the benchmarks use, directly against the
reference harness (the reference's unmodified kernels, ymgpu2d/main_ym.cu:
322-479 stage order), from the same initial state:

* 256 x 2048 (NZ x NX) with the band filter (keep |k| <= 85) and
  suppress_kz0 = 1, 3 steps: the 128-wide FCT strips with TMA bulk rows,
  the 126-column Maxwell strips, z-mean and the band filter, against the
  reference; and config 3's 1024 x 2048 with keep |k| <= NZ/3 against the
  FP64 oracle (the reference's band kernel cannot launch above NZ = 384 on
  B200).  Bar: bit for bit (the FP64 filter sums in the reference's
  warp-tree order), with the per-field relative L2 recorded beside it.
* four runs of the uneven sweep (seed 1) at NZ = 512 and 1024, alone and as
  one batch (64-wide strips, 128-row segments), 3 steps: bit for bit (two
  of them run the z-mean at NZ = 512 and 1024, where the reference needs
  its shared-memory limit raised, ymgpu2d/YM_Physics.cu:272-327).
* the 4096 x 8192 bench workload without the filter (the reference's band
  kernels cannot launch at NZ = 4096), 2 steps: bit for bit.
"""
from __future__ import annotations

import numpy as np
import pytest

from cases import BASE
from parity_report import record

pytestmark = pytest.mark.gpu

SWEEP_BASE = "alpha_YM = 1.0\nrun_mode = 6\nlx_override = 20\n"
# draws of uneven_sweep(1, 64): 1 (1024 x 2048), 4 (1024 x 256, suppress_kz0),
# 7 (512 x 512), 10 (512 x 1024, suppress_kz0)
SWEEP_DRAWS = (1, 4, 7, 10)


@pytest.fixture(scope="module")
def ref():
    from oracle import REF_PARITY_LIB, RefHarness

    if not REF_PARITY_LIB.exists():
        pytest.skip("reference harness not built")
    h = RefHarness(parity=True)
    yield h
    h.destroy()


def _ref_run(ref, cfg, nsteps):
    """Initial state and the state after nsteps of the reference's kernels."""
    from kh_simulations_b200._lib import Grid
    from kh_simulations_b200.config import derive, step_params
    from kh_simulations_b200.run import init_params

    d = derive(cfg)
    ref.create(Grid(d.nx, d.nz, d.dx, d.dz), step_params(cfg, d), raise_zmean_smem=True)
    ip, _k = init_params(cfg, d)
    ref.init(ip)
    s0 = ref.get_state()
    ref.step(nsteps)
    return s0, ref.get_state()


def _twiddles(d):
    import ctypes as C

    from kh_simulations_b200 import _lib

    mhi = max(hi for _, hi in d.bands)
    c = np.empty((mhi + 1) * d.nz, np.float32)
    s = np.empty((mhi + 1) * d.nz, np.float32)
    _lib.check(_lib.load().ymkh_twiddles(d.nz, 0, mhi, c.ctypes.data_as(C.c_void_p), s.ctypes.data_as(C.c_void_p)),
               "twiddles")
    return c.reshape(mhi + 1, d.nz), s.reshape(mhi + 1, d.nz)


def test_filtered_256x2048_vs_reference(cuda, ref):
    """The production FCT shape (128-wide strips, TMA rows at NX = 2048) with
    the band filter and z-mean, against the reference's kernels.  NZ = 256:
    the reference's band kernel (156 registers a thread, one thread per z
    cell, ymgpu2d/main_ym.cu:396) cannot launch above NZ = 384 on B200."""
    from kh_simulations_b200.config import loads
    from kh_simulations_b200.run import KHRun

    cfg = loads(BASE + "nz_override = 256\nnx_override = 2048\nkz_keep_max = 85\nsuppress_kz0 = 1\n",
                "prod_256x2048")
    n = 3
    s0, s_ref = _ref_run(ref, cfg, n)
    run = KHRun(cfg)
    assert run.fct_shape()[0] == 128  # the production strip width
    run.init()
    assert np.array_equal(run.state_numpy(), s0)
    run.step(n)
    s = run.state_numpy()
    run.close()
    rep = record("prod_256x2048_keep_kz0_vs_reference", n, s, s_ref, "keep |k| <= 85, suppress_kz0, FP64 filter")
    assert np.isfinite(s).all()
    assert np.array_equal(s, s_ref), rep


def test_filtered_1024x2048_vs_oracle(cuda, orc):
    """Config 3's grid (1024 x 2048, keep |k| <= NZ/3, suppress_kz0) with the
    FP64 filter, 2 steps, against the FP64 oracle (whose band sums follow
    the reference's warp tree); the reference's own band kernel cannot
    launch at this NZ on B200."""
    from kh_simulations_b200._lib import Grid
    from kh_simulations_b200.config import derive, loads, step_params
    from kh_simulations_b200.run import KHRun

    cfg = loads(BASE + "nz_override = 1024\nnx_override = 2048\nkz_keep_max = 341\nsuppress_kz0 = 1\n",
                "prod_1024x2048")
    d = derive(cfg)
    n = 2
    run = KHRun(cfg)
    assert run.fct_shape()[0] == 128
    run.init()
    s0 = run.state_numpy()
    run.step(n)
    s = run.state_numpy()
    run.close()
    s_orc = orc.step(Grid(d.nx, d.nz, d.dx, d.dz), step_params(cfg, d), s0.copy(), n, twiddles=_twiddles(d))
    rep = record("prod_1024x2048_keep_kz0_vs_oracle", n, s, s_orc, "keep |k| <= 341, suppress_kz0, FP64 filter")
    assert np.isfinite(s).all()
    assert np.array_equal(s, s_orc), rep


def test_uneven_sweep_draws_vs_reference(cuda, ref):
    import torch

    from kh_simulations_b200.batch import KHBatch
    from kh_simulations_b200.run import KHRun
    from kh_simulations_b200.server import uneven_sweep

    cfgs = uneven_sweep(1, 64, SWEEP_BASE)
    n = 3
    st = torch.cuda.Stream()
    batch = KHBatch()
    expect, alone, members = [], [], []
    for i in SWEEP_DRAWS:
        s0, s_ref = _ref_run(ref, cfgs[i], n)
        expect.append(s_ref)
        r = KHRun(cfgs[i])
        r.init()
        assert np.array_equal(r.state_numpy(), s0), i
        r.step(n)
        alone.append(r.state_numpy())
        r.close()
        m = KHRun(cfgs[i])
        m.init()
        batch.add(m)
        members.append(m)
    batch.step(n, st)
    st.synchronize()
    batch.check(st)
    for i, e, a, m in zip(SWEEP_DRAWS, expect, alone, members):
        assert np.array_equal(a, e), (i, np.abs(a - e).max())
        assert np.array_equal(m.state_numpy(), e), i
    batch.close()
    for m in members:
        m.close()


def test_bench_workload_one_step_vs_reference(cuda, ref):
    """4096 x 8192, filter off: 2 steps bit for bit against the reference
    (about 40 GB of device memory for the reference's arrays and 13 GB for
    the run's two buffers)."""
    import torch

    from kh_simulations_b200.config import loads
    from kh_simulations_b200.run import KHRun

    cfg = loads(BASE + "nz_override = 4096\nnx_override = 8192\n", "kh_4096x8192")
    n = 2
    s0, s_ref = _ref_run(ref, cfg, n)
    ref.destroy()
    run = KHRun(cfg)
    run.init()
    torch.cuda.synchronize()
    for i in range(24):
        assert np.array_equal(run.state[i].cpu().numpy(), s0[i]), ("init", i)
    del s0
    run.step(n)
    torch.cuda.synchronize()
    for i in range(24):
        got = run.state[i].cpu().numpy()
        assert np.array_equal(got, s_ref[i]), (i, np.abs(got - s_ref[i]).max())
    run.close()
    torch.cuda.empty_cache()
