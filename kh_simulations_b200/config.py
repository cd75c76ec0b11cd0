"""The reference's ``.ini`` run configuration and the quantities derived from it.

``RunConfig`` mirrors ``struct RunConfig`` (ymgpu2d/YM_Config.cuh:6-49) key
for key with the same defaults; ``load_config`` follows
``load_config`` (ymgpu2d/YM_Config.cu:15-136): ``#`` comment lines, inline
``#`` comments stripped, unknown keys only warn, float keys parsed with the C
library's ``strtof`` (what ``std::stof`` calls) so values are rounded to
float exactly as the reference rounds them, and the same constraint checks.
``derive`` reproduces the grid/parameter derivation of ymgpu2d/main_ym.cu:51-83
and the run-length/stride rules of :244-249.

Extension keys (not in the reference; they never change the step itself):
  ``kz_keep_max = K``   subtract modes (K, NZ/2] every step (keep |k| <= K)
  ``kz_bands = a-b,c-d`` explicit extra subtraction bands
  ``filter_engine = dft | tf32x3``  how the band filter runs: FP64 sums with
                        the reference's FP32 twiddles (default), or the
                        tensor cores with 3-pass split TF32
"""
from __future__ import annotations

import ctypes
import math
import sys
import warnings
from dataclasses import dataclass, field, fields
from pathlib import Path

_libc = ctypes.CDLL(None)
_libc.strtof.restype = ctypes.c_float
_libc.strtof.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_char_p)]
_libc.strtol.restype = ctypes.c_long
_libc.strtol.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_char_p), ctypes.c_int]


def stof(text: str) -> float:
    """std::stof: strtof on the longest numeric prefix; error if none."""
    b = text.encode()
    end = ctypes.c_char_p()
    v = _libc.strtof(b, ctypes.byref(end))
    consumed = len(b) - len(end.value or b"")
    if consumed == 0:
        raise ValueError(f"stof: no conversion: {text!r}")
    return float(v)


def stoi(text: str) -> int:
    """std::stoi: strtol base 10 on the longest numeric prefix; error if none."""
    b = text.encode()
    end = ctypes.c_char_p()
    v = _libc.strtol(b, ctypes.byref(end), 10)
    consumed = len(b) - len(end.value or b"")
    if consumed == 0:
        raise ValueError(f"stoi: no conversion: {text!r}")
    if not -(2**31) <= v < 2**31:
        raise ValueError(f"stoi: out of range: {text!r}")
    return int(v)


def f32(x: float) -> float:
    """Round a Python float to the nearest float32 (a C `float` literal)."""
    return float(ctypes.c_float(x).value)


@dataclass
class RunConfig:
    """struct RunConfig, ymgpu2d/YM_Config.cuh:6-49 (float fields hold float32 values)."""

    k_mode: int = 1
    alpha_YM: float = f32(0.5)
    perturb_amp: float = f32(0.001)
    run_mode: int = 6
    V0: float = f32(0.1)
    xi_sponge: float = 0.0
    sigma_sponge: float = 5.0
    xi_cut: float = 0.0
    warm_T: float = 0.0
    freeze_override: int = -1
    suppress_kz0: int = 0
    hyp_diff: float = 0.0
    kz_suppress_max: int = 0
    eps_override: float = -1.0
    kz_suppress_hi: int = 0
    vz_edge_taper: float = 0.0
    init_by1_eq: int = 0
    nz_override: int = -1
    nx_override: int = -1
    courant_override: float = -1.0
    lz_override: float = -1.0
    lx_override: float = -1.0
    target_tu: float = -1.0
    run_tag: str = ""
    seed_profile_file: str = ""
    # extensions
    kz_keep_max: int = -1
    kz_bands: list = field(default_factory=list)
    filter_engine: str = "dft"
    eigen_seed: int = 0       # 1: seed from the eigenmode solved at init (no seed file)
    eigen_seed_nx: int = 384  # grid of that solve (the reference solver's default)


FILTER_ENGINES = {"dft": 0, "tf32x3": 1}

_INT_KEYS = {"k_mode", "run_mode", "freeze_override", "suppress_kz0", "kz_suppress_max", "kz_suppress_hi",
             "init_by1_eq", "nz_override", "nx_override", "kz_keep_max", "eigen_seed", "eigen_seed_nx"}
_STR_KEYS = {"run_tag", "seed_profile_file", "filter_engine"}
_FLOAT_KEYS = {f.name for f in fields(RunConfig)} - _INT_KEYS - _STR_KEYS - {"kz_bands"}


class ConfigError(ValueError):
    pass


def parse_bands(text: str) -> list:
    out = []
    for part in text.split(","):
        part = part.strip()
        if not part:
            continue
        lo, _, hi = part.partition("-")
        out.append((stoi(lo), stoi(hi or lo)))
    return out


def loads(text: str, path: str = "<string>") -> RunConfig:
    """Parse .ini text (ymgpu2d/YM_Config.cu:26-73) and validate (:203-217)."""
    cfg = RunConfig()
    for lineno, raw in enumerate(text.splitlines(), 1):
        line = raw.strip(" \t\r\n")
        if not line or line.startswith("#"):
            continue
        if "=" not in line:
            warnings.warn(f"{path}:{lineno}: no '=' found, skipping: {line}")
            continue
        key, _, val = line.partition("=")
        key = key.strip(" \t\r\n")
        val = val.strip(" \t\r\n")
        if "#" in val:
            val = val[: val.index("#")].strip(" \t\r\n")
        if key in _INT_KEYS:
            setattr(cfg, key, stoi(val))
        elif key in _FLOAT_KEYS:
            setattr(cfg, key, stof(val))
        elif key in _STR_KEYS:
            setattr(cfg, key, val)
        elif key == "kz_bands":
            cfg.kz_bands = parse_bands(val)
        else:
            warnings.warn(f"{path}:{lineno}: unknown key '{key}'")
    validate(cfg)
    return cfg


def load_config(path: str | Path) -> RunConfig:
    p = Path(path)
    try:
        text = p.read_text()
    except OSError as e:
        raise ConfigError(f"cannot open config file '{p}'") from e
    return loads(text, str(p))


def grid_size(cfg: RunConfig) -> tuple:
    nz = cfg.nz_override if cfg.nz_override > 0 else 64
    nx = cfg.nx_override if cfg.nx_override > 0 else 768
    return nx, nz


def validate(cfg: RunConfig) -> None:
    """Constraint checks of ymgpu2d/YM_Config.cu:203-211."""
    nx, nz = grid_size(cfg)
    if cfg.suppress_kz0 and (nz & (nz - 1)) != 0:
        raise ConfigError(f"suppress_kz0=1 requires NZ to be a power of 2 (got NZ={nz})")
    if (cfg.kz_suppress_max >= 1 or cfg.kz_suppress_hi > 0) and nz % 32 != 0:
        raise ConfigError(f"kz_suppress_max/kz_suppress_hi require NZ multiple of 32 (got NZ={nz})")
    if cfg.lz_override > 0 and cfg.nz_override < 0:
        warnings.warn(f"lz_override set but nz_override not set (NZ={nz})")
    if cfg.lx_override > 0 and cfg.nx_override < 0:
        warnings.warn(f"lx_override set but nx_override not set (NX={nx})")


@dataclass
class Derived:
    """Grid, step parameters and loop controls of ymgpu2d/main_ym.cu:51-83, 244-249."""

    nx: int
    nz: int
    lx: float
    lz: float
    dx: float
    dz: float
    courant: float
    dt: float
    V0: float
    eps: float
    alpha: float
    freeze_az1: int
    periodic_x: int
    total_steps: int
    export_stride: int
    energy_stride: int
    energy_thresh: float
    bands: list  # (lo, hi) in application order


def derive(cfg: RunConfig) -> Derived:
    nx, nz = grid_size(cfg)
    lx = cfg.lx_override if cfg.lx_override > 0 else 6.0 * math.pi
    lz = cfg.lz_override if cfg.lz_override > 0 else 2.0 * math.pi
    dx = lx / nx
    dz = lz / nz
    courant = cfg.courant_override if cfg.courant_override > 0 else f32(0.1)
    dt = courant * dx
    eps = cfg.eps_override if cfg.eps_override > 0 else lx / 6.0
    freeze = 1 if cfg.run_mode in (1, 3, 4, 5, 6) else 0
    if cfg.freeze_override >= 0:
        freeze = cfg.freeze_override
    periodic = 1 if cfg.run_mode >= 1 else 0
    if cfg.target_tu > 0:
        total = int(cfg.target_tu / dt)
        export_stride = max(1, int(1.0 / dt))
        energy_stride = max(1, int(0.5 / dt))
    else:
        total, export_stride, energy_stride = 2000000, 20000, 10000
    thresh = 100.0 if (cfg.run_mode >= 3 or cfg.xi_sponge > 0) else 5.0
    bands = []
    if cfg.kz_suppress_max >= 1:
        bands.append((1, cfg.kz_suppress_max))
    if cfg.kz_suppress_hi > cfg.kz_suppress_max + 1:
        bands.append((cfg.kz_suppress_max + 2, cfg.kz_suppress_hi))
    extra = list(cfg.kz_bands)
    if cfg.kz_keep_max >= 0 and cfg.kz_keep_max < nz // 2:
        extra.append((cfg.kz_keep_max + 1, nz // 2))
    bands.extend(extra)
    return Derived(nx, nz, lx, lz, dx, dz, courant, dt, cfg.V0, eps, cfg.alpha_YM, freeze, periodic,
                   total, export_stride, energy_stride, thresh, bands)


def step_params(cfg: RunConfig, d: Derived | None = None):
    """ymkh_params for the C ABI (main_ym.cu:67-83 plus the extension bands)."""
    from ._lib import MAX_EXTRA_BANDS, Params

    d = d or derive(cfg)
    p = Params()
    p.dx, p.dz, p.dt_step = d.dx, d.dz, d.dt
    p.c, p.eps_0 = 1.0, 1.0
    p.alpha_YM = d.alpha
    p.V0, p.epsilon = d.V0, d.eps
    p.freeze_az1, p.periodic_x = d.freeze_az1, d.periodic_x
    p.xi_sponge, p.sigma_sponge, p.xi_cut = cfg.xi_sponge, cfg.sigma_sponge, cfg.xi_cut
    p.warm_T = cfg.warm_T
    p.suppress_kz0 = cfg.suppress_kz0
    p.hyp_diff_coeff = cfg.hyp_diff
    p.kz_suppress_max, p.kz_suppress_hi = cfg.kz_suppress_max, cfg.kz_suppress_hi
    extra = d.bands[(1 if cfg.kz_suppress_max >= 1 else 0) + (1 if cfg.kz_suppress_hi > cfg.kz_suppress_max + 1 else 0):]
    if len(extra) > MAX_EXTRA_BANDS:
        raise ConfigError(f"at most {MAX_EXTRA_BANDS} extra bands")
    p.n_extra_bands = len(extra)
    for i, (lo, hi) in enumerate(extra):
        p.extra_band_lo[i], p.extra_band_hi[i] = lo, hi
    if cfg.filter_engine not in FILTER_ENGINES:
        raise ConfigError(f"filter_engine must be one of {sorted(FILTER_ENGINES)}, got {cfg.filter_engine!r}")
    p.filter_engine = FILTER_ENGINES[cfg.filter_engine]
    return p


def out_dir_name(cfg: RunConfig, d: Derived | None = None) -> str:
    """Output directory name of ymgpu2d/main_ym.cu:143-170."""
    d = d or derive(cfg)
    tags = {1: "_circ", 2: "_emhd", 3: "_dtanh", 4: "_step", 5: "_tanh", 6: "_circ_az2seed"}
    s = f"ym_k{cfg.k_mode}_a{cfg.alpha_YM:.3f}"
    if cfg.perturb_amp == 0.0:
        s += "_noperturb"
    s += tags.get(cfg.run_mode, "")
    if cfg.V0 != 0.1:
        s += f"_v{cfg.V0:.4f}"
    if cfg.xi_sponge > 0.0:
        s += f"_sp{cfg.xi_sponge:.1f}"
    if cfg.xi_cut > 0.0:
        s += f"_xc{cfg.xi_cut:.1f}"
    if d.freeze_az1 and cfg.run_mode == 0:
        s += "_frz"
    if cfg.eps_override > 0.0:
        s += f"_eps{cfg.eps_override:.2f}"
    if cfg.nx_override > 0:
        s += f"_nx{cfg.nx_override}"
    if cfg.lx_override > 0:
        s += f"_lx{cfg.lx_override:.2f}"
    if cfg.suppress_kz0:
        s += "_nkz0"
    if cfg.kz_suppress_max >= 1:
        s += f"_nkz1to{cfg.kz_suppress_max}"
    if cfg.kz_suppress_hi > 0:
        s += f"_bp{cfg.kz_suppress_hi}"
    if cfg.hyp_diff > 0.0:
        s += f"_hd{cfg.hyp_diff:.0e}"
    if cfg.run_tag:
        s += "_" + cfg.run_tag
    return s


if __name__ == "__main__":  # pragma: no cover
    c = load_config(sys.argv[1])
    print(c)
    print(derive(c))
