"""ctypes binding of the in-tree CUDA library (include/ymkh.h).

The library must be present: there is no CPU fallback.  A missing or
unloadable ``libymkh.so`` raises ``YMKHError`` at first use.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

_PKG = Path(__file__).resolve().parent
LIB_PATH = _PKG / "libymkh.so"
DEBUG_LIB_PATH = _PKG / "libymkh_debug.so"  # the same library with checked accesses (YMKH_DEBUG)

NFIELDS, NFLUID, NSTATE = 12, 6, 24
MAX_EXTRA_BANDS = 4
NOALLOC_MAX_CELLS = 134217728  # YMKH_NOALLOC_MAX_CELLS
FILTER_DFT, FILTER_TF32X3 = 0, 1
FCT_FUSED, FCT_SPLIT = 0, 1
YMKH_BUILD_DEBUG = 1  # ymkh_build_flags(): the library's kernels check their accesses
ERR_WAIT, ERR_BOUNDS = 1, 2  # bits of the device error word
PAIRS = {"Az": 0, "By": 1, "Ex": 2, "Ez": 3}  # YMKH_PAIR_*
GAUSS_NOUT = 16  # YMKH_GAUSS_NOUT
SNAP_CSV, SNAP_FP64 = 0, 1

# state order of include/ymkh.h
STATE_NAMES = (
    "Ex1", "Ex2", "Ex3", "Ez1", "Ez2", "Ez3", "By1", "By2", "By3", "Az1", "Az2", "Az3",
    "nA", "pxA", "pzA", "Q1A", "Q2A", "Q3A",
    "nB", "pxB", "pzB", "Q1B", "Q2B", "Q3B",
)


class YMKHError(RuntimeError):
    pass


class Grid(C.Structure):
    _fields_ = [("nx", C.c_int), ("nz", C.c_int), ("dx", C.c_double), ("dz", C.c_double)]


class Params(C.Structure):
    """ymkh_params: YMParams (ymgpu2d/YM_Physics.cuh:31-46) plus extensions."""

    _fields_ = [
        ("dx", C.c_double), ("dz", C.c_double), ("dt_step", C.c_double),
        ("c", C.c_double), ("eps_0", C.c_double),
        ("alpha_YM", C.c_double),
        ("V0", C.c_double), ("epsilon", C.c_double),
        ("freeze_az1", C.c_int), ("periodic_x", C.c_int),
        ("xi_sponge", C.c_double), ("sigma_sponge", C.c_double), ("xi_cut", C.c_double),
        ("warm_T", C.c_double),
        ("suppress_kz0", C.c_int),
        ("hyp_diff_coeff", C.c_double),
        ("kz_suppress_max", C.c_int), ("kz_suppress_hi", C.c_int),
        ("n_extra_bands", C.c_int),
        ("extra_band_lo", C.c_int * MAX_EXTRA_BANDS),
        ("extra_band_hi", C.c_int * MAX_EXTRA_BANDS),
        ("filter_engine", C.c_int),
    ]


class InitParams(C.Structure):
    _fields_ = [
        ("run_mode", C.c_int), ("k_mode", C.c_int),
        ("perturb_amp", C.c_double), ("V0", C.c_double), ("epsilon", C.c_double),
        ("alpha_YM", C.c_double), ("init_by1_eq", C.c_int), ("vz_edge_taper", C.c_double),
        ("seed_by", C.c_void_p), ("seed_ex", C.c_void_p), ("seed_ez", C.c_void_p),
        ("seed_az", C.c_void_p), ("seed_qA", C.c_void_p), ("seed_qB", C.c_void_p),
    ]


_lib = None

_SIGS = {
    "ymkh_last_error": (C.c_int, [C.c_char_p, C.c_size_t]),
    "ymkh_create": (C.c_int, [C.POINTER(Grid), C.POINTER(Params), C.POINTER(C.c_void_p)]),
    "ymkh_set_params": (C.c_int, [C.c_void_p, C.POINTER(Params)]),
    "ymkh_bind_state": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), C.POINTER(C.c_void_p)]),
    "ymkh_bind_state2": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p)]),
    "ymkh_current_buffer": (C.c_int, [C.c_void_p]),
    "ymkh_set_current_buffer": (C.c_int, [C.c_void_p, C.c_int]),
    "ymkh_set_graph_steps": (C.c_int, [C.c_void_p, C.c_int]),
    "ymkh_set_fct_shape": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    "ymkh_get_fct_shape": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "ymkh_set_fct_mode": (C.c_int, [C.c_void_p, C.c_int]),
    "ymkh_batch_set_fct_mode": (C.c_int, [C.c_void_p, C.c_int]),
    "ymkh_init": (C.c_int, [C.c_void_p, C.POINTER(InitParams), C.c_void_p]),
    "ymkh_step": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "ymkh_energy": (C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.c_void_p]),
    "ymkh_energy_async": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "ymkh_mode_amp": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_double), C.c_void_p]),
    "ymkh_circ_amp": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.POINTER(C.c_double), C.c_void_p]),
    "ymkh_gauss": (C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.c_void_p]),
    "ymkh_snapshot": (C.c_int, [C.c_void_p, C.c_char_p, C.c_int, C.c_void_p]),
    "ymkh_snapshot_wait": (C.c_int, [C.c_void_p]),
    "ymkh_destroy": (C.c_int, [C.c_void_p]),
    "ymkh_check": (C.c_int, [C.c_void_p, C.c_void_p]),
    "ymkh_batch_create": (C.c_int, [C.POINTER(C.c_void_p)]),
    "ymkh_batch_add": (C.c_int, [C.c_void_p, C.c_void_p]),
    "ymkh_batch_remove": (C.c_int, [C.c_void_p, C.c_void_p]),
    "ymkh_batch_size": (C.c_int, [C.c_void_p]),
    "ymkh_batch_set_graph_steps": (C.c_int, [C.c_void_p, C.c_int]),
    "ymkh_batch_step": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "ymkh_batch_check": (C.c_int, [C.c_void_p, C.c_void_p]),
    "ymkh_batch_destroy": (C.c_int, [C.c_void_p]),
    "ymkh_twiddles": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p]),
    "ymkh_launch_count": (C.c_longlong, []),
    "ymkh_build_flags": (C.c_int, []),
    "ymkh_energy_noalloc": (C.c_int, [C.POINTER(C.c_void_p), C.c_int, C.c_int, C.c_void_p, C.c_void_p]),
    "ymkh_stage_times": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.POINTER(C.c_float), C.c_int]),
}

STAGES = ("fct", "maxwell", "sponge_xicut", "zmean", "bands", "hyperdiff", "zero_colour1")

# Symbols every build must export (checked by the CPU test suite).
EXPORTED = tuple(_SIGS)


def load(path: Path | str | None = None):
    """Load libymkh.so (once) and declare the signatures."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise YMKHError(f"CUDA library not built: {p} (run python -m kh_simulations_b200.build)")
    try:
        lib = C.CDLL(str(p))
    except OSError as e:  # pragma: no cover - depends on the host
        raise YMKHError(f"cannot load {p}: {e}") from e
    for name, (res, args) in _SIGS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


def last_error() -> str:
    buf = C.create_string_buffer(512)
    load().ymkh_last_error(buf, 512)
    return buf.value.decode(errors="replace")


def check(rc: int, what: str) -> None:
    if rc != 0:
        raise YMKHError(f"{what} failed ({rc}): {last_error()}")


def launch_count() -> int:
    return int(load().ymkh_launch_count())
