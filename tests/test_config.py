"""The .ini layer follows ymgpu2d/YM_Config.cu and main_ym.cu:51-83."""
import math
import warnings

import numpy as np
import pytest

from kh_simulations_b200.config import ConfigError, derive, f32, loads, out_dir_name, stof, stoi

INI = """
# comment line
k_mode          = 1          # integer z-mode
alpha_YM        = 2.0        # SU(2) colour coupling
perturb_amp     = 0.001
run_mode        = 6
V0              = 0.05       # shear velocity
xi_sponge       = 13.0
sigma_sponge    = 5.0
warm_T          = 0.0
suppress_kz0    = 1
hyp_diff        = 5e-5
kz_suppress_max = 0
eps_override    = 0.15
kz_suppress_hi  = 14
nz_override     = 128
lz_override     = 12.5664
target_tu       = 100
"""


def test_float_keys_are_float_rounded():
    cfg = loads(INI)
    assert cfg.V0 == float(np.float32(0.05)) and cfg.V0 != 0.05
    assert cfg.eps_override == float(np.float32(0.15))
    assert cfg.hyp_diff == float(np.float32(5e-5))
    assert cfg.lz_override == float(np.float32(12.5664))
    assert cfg.kz_suppress_hi == 14 and cfg.suppress_kz0 == 1


def test_derivation_matches_main():
    cfg = loads(INI)
    d = derive(cfg)
    assert (d.nx, d.nz) == (768, 128)
    assert d.lx == 6.0 * math.pi and d.lz == float(np.float32(12.5664))
    assert d.dx == d.lx / 768 and d.dz == d.lz / 128
    assert d.courant == float(np.float32(0.1))
    assert d.dt == d.courant * d.dx
    assert d.freeze_az1 == 1 and d.periodic_x == 1
    assert d.total_steps == int(float(np.float32(100.0)) / d.dt)
    assert d.energy_stride == max(1, int(0.5 / d.dt))
    assert d.energy_thresh == 100.0  # sponge on
    assert d.bands == [(2, 14)]
    assert out_dir_name(cfg).startswith("ym_k1_a2.000_circ_az2seed_v0.0500_sp13.0_eps0.15_nkz0_bp14_hd5e-05")


def test_stof_stoi_prefix_semantics():
    assert stof("0.15abc") == f32(0.15)
    assert stoi("12 ") == 12
    with pytest.raises(ValueError):
        stof("abc")
    with pytest.raises(ValueError):
        loads("k_mode = x\n")


def test_unknown_key_warns_and_constraints_raise():
    with warnings.catch_warnings(record=True) as w:
        warnings.simplefilter("always")
        loads("nonsense = 3\n")
        assert any("unknown key" in str(x.message) for x in w)
    with pytest.raises(ConfigError):
        loads("suppress_kz0 = 1\nnz_override = 96\n")
    with pytest.raises(ConfigError):
        loads("kz_suppress_hi = 5\nnz_override = 100\n")


def test_defaults_and_extension_bands():
    d = derive(loads(""))
    assert (d.nx, d.nz) == (768, 64) and d.periodic_x == 1 and d.bands == []
    d = derive(loads("nz_override = 256\nkz_keep_max = 85\nkz_bands = 3-4, 9\n"))
    assert d.bands == [(3, 4), (9, 9), (86, 128)]
    d = derive(loads("run_mode = 0\n"))
    assert d.periodic_x == 0 and d.freeze_az1 == 0 and d.energy_thresh == 5.0


def test_filter_engine_key():
    """Extension key `filter_engine` selects the band filter engine of the
    C ABI (YMKH_FILTER_DFT = 0, YMKH_FILTER_TF32X3 = 1); other values are
    rejected when the step parameters are formed."""
    import pytest

    from kh_simulations_b200.config import ConfigError, loads, step_params

    base = "nz_override = 128\nnx_override = 256\nkz_keep_max = 42\n"
    assert step_params(loads(base)).filter_engine == 0
    assert step_params(loads(base + "filter_engine = tf32x3\n")).filter_engine == 1
    with pytest.raises(ConfigError):
        step_params(loads(base + "filter_engine = fp16\n"))
