"""Eigenmode-seeded runs on the GPU.

- ``eigen_seed = 1`` gives the state that the same profiles give through a
  seed file, bit for bit: the in-process seed is a seed file without the
  file.
- Physics pin: the kz = 1, alpha = 1, V0 = 0.05, EPS = 0.15 mode with the
  sponge at xi = 20 has gamma = 0.08967 on the solver's grid (0.08969 at
  NX = 768, the value of ymgpu2d/eigenmode_kz1_a1.00_V0.05_EPS0.15.npz).
  Seeded with it on the reference's production grid (NZ 64, NX 768,
  Courant 0.1) with its campaign filters (z-mean removal, modes 2..14
  subtracted, hyperdiffusion 5e-5), a 60 TU run grows at the rate that
  the reference's analysis fits to |Az2 + i Az3| (batch_analyze.py), within
  GAMMA_RTOL of the eigenvalue (measured on a B200: 0.0889, 0.9% below;
  the 256 x 768 grid at Courant 0.01 gives the same).
"""
import numpy as np
import pytest

from kh_simulations_b200 import eigenmode as em
from kh_simulations_b200 import growth
from kh_simulations_b200.config import loads
from kh_simulations_b200.run import KHRun
from kh_simulations_b200.seed import write_seed

pytestmark = pytest.mark.gpu

GAMMA_RTOL = 0.02
INI = ("k_mode = 1\nalpha_YM = 1.0\nV0 = 0.05\nperturb_amp = 0.001\nrun_mode = 6\nxi_sponge = 20\n"
       "sigma_sponge = 5\neps_override = 0.15\neigen_seed = 1\nsuppress_kz0 = 1\nhyp_diff = 5e-5\n"
       "kz_suppress_max = 0\nkz_suppress_hi = 14\nnz_override = 64\nnx_override = 768\n"
       "courant_override = 0.1\ntarget_tu = 60\n")


def test_eigen_seed_equals_its_seed_file(tmp_path):
    cfg = loads(INI, "eig")
    a = KHRun(cfg)
    a.init()
    prof = em.cached_seed(em.spec_for_run(cfg, a.d, cfg.eigen_seed_nx))
    write_seed(tmp_path / em.seed_file_name(em.spec_for_run(cfg, a.d)), prof)
    b = KHRun(cfg)
    b.init(seed_file=tmp_path / em.seed_file_name(em.spec_for_run(cfg, a.d)))
    sa, sb = a.state_numpy(), b.state_numpy()
    assert np.array_equal(sa.view(np.uint64), sb.view(np.uint64))
    assert np.abs(sa[11]).max() > 0  # Az3 carries the seeded mode
    a.close()
    b.close()


def test_seeded_run_grows_at_the_eigenvalue():
    cfg = loads(INI, "eig")
    run = KHRun(cfg)
    run.init()
    gamma = em.solve(em.spec_for_run(cfg, run.d, cfg.eigen_seed_nx)).gamma.real
    t, amp = [], []
    run.run(on_export=lambda r, s: (t.append(s * r.d.dt), amp.append(r.circ_amp("Az")[0])))
    assert not run.halted, run.halt_reason
    g, t0, t1, r2 = growth.fit_growth_rate(np.array(t), np.array(amp))
    print(f"eigenvalue {gamma:.5f}, fitted {g:.5f} over [{t0:.1f}, {t1:.1f}], R2 {r2:.5f}")
    assert r2 > 0.999
    assert g == pytest.approx(gamma, rel=GAMMA_RTOL)
    run.close()
