"""Eigenmode seeds against the reference's own solver (CPU).

tests/golden/eigen_seeds.npz (tests/golden/make_eigen_fixtures.py) holds,
for nine parameter sets, what ymgpu2d/analysis/ym_eigenmode.py computes
(where two eigenvalues tie on growth, the one with positive imaginary part):
the chosen eigenvalue, the eigenvalues near the shift and the float32 seed
profiles.  Six of them equal the seed files the reference ships
(ymgpu2d/seeds/) to float32 rounding, which the generating script checked.
ARPACK starts from a random vector, so two solves agree to its tolerance
(1e-10), not bit for bit: eigenvalues are compared to 1e-9 and profiles,
which are normalised to a peak of 1, to 2e-5 (two runs of the reference's
solver itself differ by up to 5.8e-6 in one of these cases).
"""
import math

import numpy as np
import pytest

from kh_simulations_b200 import eigenmode as em
from kh_simulations_b200.seed import FIELD_ORDER, read_seed, write_seed

FIX = np.load(__import__("pathlib").Path(__file__).parent / "golden" / "eigen_seeds.npz")
CASES = list(range(int(FIX["ncases"])))


def _spec(c):
    k, alpha, v0, eps, nx, lx, lz, xsp, xcut = FIX[f"case{c}_params"]
    return em.ModeSpec(int(k), float(alpha), float(v0), float(eps), int(nx), float(lx), float(lz), float(xsp),
                       xi_cut=None if xcut < 0 else float(xcut))


@pytest.mark.parametrize("c", CASES)
def test_mode_matches_the_reference_solver(c):
    spec = _spec(c)
    mode = em.solve(spec)
    ref_g = complex(FIX[f"case{c}_gamma"])
    assert abs(mode.gamma - ref_g) <= 1e-9 * abs(ref_g)
    got = np.stack([mode.seed_profiles()[k] for k in FIELD_ORDER])
    assert np.abs(got - FIX[f"case{c}_profiles"]).max() < 2e-5
    # the eigenvalues found near the shift include the chosen one both times
    assert np.abs(FIX[f"case{c}_eigenvalues"] - mode.gamma).min() <= 1e-9 * abs(ref_g)
    name = str(FIX[f"case{c}_name"])
    if name:
        assert em.seed_file_name(spec) == name


def test_growth_rate_of_the_reference_eigenmode_file():
    """ymgpu2d/eigenmode_kz1_a1.00_V0.05_EPS0.15.npz (NX 768, sponge at
    xi = 20) holds gamma = 0.08969; case 8 is that problem."""
    g = em.solve(_spec(8)).gamma
    assert abs(g - complex(FIX["npz_gamma"])) < 1e-9


def test_seed_file_round_trip(tmp_path):
    mode = em.solve(_spec(0))
    prof = mode.seed_profiles()
    write_seed(tmp_path / "s.bin", prof)
    back = read_seed(tmp_path / "s.bin")
    for k in FIELD_ORDER:
        assert np.array_equal(back[k], prof[k])


def test_solve_many_in_worker_processes():
    specs = [_spec(0), _spec(4)]
    got = em.solve_many(specs, workers=2)
    for s, (g, prof) in zip(specs, got):
        one = em.solve(s)
        assert abs(g - one.gamma) <= 1e-9 * abs(one.gamma)
        assert np.abs(prof["az"] - one.seed_profiles()["az"]).max() < 2e-5


def test_wkb_shift():
    assert em.wkb_gamma(1.0, 1.0, 0.05) == pytest.approx(0.2179614359949621, rel=1e-12)
    assert math.isnan(em.wkb_gamma(1.0, 0.0, 0.05))


def test_run_parameters_give_the_reference_seed():
    """An .ini with eigen_seed = 1 solves the problem the reference's seed
    file eigenmode_seed_kz1_a1.00_V0.050_sp20.0.bin was made for (case 0):
    float32 .ini values go to the solver as their decimals."""
    from kh_simulations_b200.config import derive, loads

    cfg = loads("k_mode = 1\nalpha_YM = 1.0\nV0 = 0.05\neps_override = 0.15\nxi_sponge = 20\n"
                "sigma_sponge = 5\neigen_seed = 1\nnz_override = 64\nnx_override = 768\n", "e")
    spec = em.spec_for_run(cfg, derive(cfg), cfg.eigen_seed_nx)
    assert spec == _spec(0)
    prof = em.cached_seed(spec)
    got = np.stack([prof[k] for k in FIELD_ORDER])
    assert np.abs(got - FIX["case0_profiles"]).max() < 2e-5
