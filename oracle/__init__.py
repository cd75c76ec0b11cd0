"""Checkers for the CUDA path — TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline/reference
legs may import this package.  It never stands in for the product path.

  Oracle      libymoracle.so: FP64 OpenMP CPU restatement of the reference
              step (ym_oracle.cpp), in the reference's operation order.
  RefHarness  oracle/_ref/libymref*.so: the reference's own kernels compiled
              unmodified from its sources (ref_harness.cu + Makefile), on GPU.

build() compiles both (the _ref part only where the reference tree exists).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_LIB = HERE / "libymoracle.so"
REF_PARITY_LIB = HERE / "_ref" / "libymref_parity.so"
REF_STOCK_LIB = HERE / "_ref" / "libymref.so"
# The reference's ymgpu2d tree for the _ref targets: $YMKH_REFERENCE_DIR, else
# the location the Makefile recipe names (absent on machines without it).
REF_DIR = os.environ.get("YMKH_REFERENCE_DIR")

NSTATE = 24


def build(ref: bool = True) -> None:
    targets = ["oracle"] + (["ref"] if ref else [])  # the recipe skips _ref when the tree is absent
    subprocess.run(["make", "-s", "-C", str(HERE), *targets, *([f"REF_DIR={REF_DIR}"] if REF_DIR else [])],
                   check=True)


def _ptrs(state: np.ndarray):
    assert state.dtype == np.float64 and state.flags.c_contiguous and state.shape[0] == NSTATE
    return (C.c_void_p * NSTATE)(*[state[i].ctypes.data for i in range(NSTATE)])


class Oracle:
    """ctypes wrapper of libymoracle.so."""

    def __init__(self, path: Path | str = ORACLE_LIB):
        from kh_simulations_b200._lib import Grid, Params

        if not Path(path).exists():
            build(ref=False)
        self.lib = C.CDLL(str(path))
        self.Grid, self.Params = Grid, Params
        self.lib.orc_step.restype = C.c_int
        PP = C.POINTER(C.c_void_p)
        self.lib.orc_step.argtypes = [C.POINTER(Grid), C.POINTER(Params), PP, C.c_int, C.c_void_p, C.c_void_p,
                                      C.c_int]
        self.lib.orc_energy.restype = C.c_double
        self.lib.orc_energy.argtypes = [C.POINTER(Grid), PP]
        self.lib.orc_mode_amp.restype = C.c_int
        self.lib.orc_mode_amp.argtypes = [C.POINTER(Grid), PP, C.c_int, C.POINTER(C.c_double)]
        self.lib.orc_twiddles.restype = C.c_int
        self.lib.orc_twiddles.argtypes = [C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p]
        self.lib.orc_num_threads.restype = C.c_int

    def threads(self) -> int:
        return int(self.lib.orc_num_threads())

    def step(self, grid, params, state: np.ndarray, nsteps: int = 1, twiddles=None) -> np.ndarray:
        """Advance `state` ([24, NZ, NX] float64, C order) in place."""
        tc = ts = None
        mmax = -1
        if twiddles is not None:
            tc, ts = (np.ascontiguousarray(t, dtype=np.float32) for t in twiddles)
            mmax = tc.shape[0] - 1
        rc = self.lib.orc_step(C.byref(grid), C.byref(params), _ptrs(state), int(nsteps),
                               tc.ctypes.data if tc is not None else None,
                               ts.ctypes.data if ts is not None else None, mmax)
        if rc:
            raise RuntimeError(f"orc_step failed ({rc})")
        return state

    def energy(self, grid, state: np.ndarray) -> float:
        return float(self.lib.orc_energy(C.byref(grid), _ptrs(state)))

    def mode_amp(self, grid, state: np.ndarray, k: int) -> tuple:
        out = (C.c_double * 2)()
        self.lib.orc_mode_amp(C.byref(grid), _ptrs(state), int(k), out)
        return out[0], out[1]

    def twiddles(self, nz: int, m_lo: int, m_hi: int) -> tuple:
        n = (m_hi - m_lo + 1) * nz
        c = np.empty(n, np.float32)
        s = np.empty(n, np.float32)
        self.lib.orc_twiddles(nz, m_lo, m_hi, c.ctypes.data, s.ctypes.data)
        return c.reshape(-1, nz), s.reshape(-1, nz)


class RefHarness:
    """ctypes wrapper of the reference-kernel harness (one live instance per process)."""

    def __init__(self, parity: bool = True):
        from kh_simulations_b200._lib import Grid, InitParams, Params

        path = REF_PARITY_LIB if parity else REF_STOCK_LIB
        if not path.exists():
            raise FileNotFoundError(f"{path} not built (make -C oracle ref)")
        self.lib = C.CDLL(str(path))
        L = self.lib
        L.ymref_last_error.restype = C.c_char_p
        L.ymref_create.argtypes = [C.POINTER(Grid), C.POINTER(Params), C.c_int]
        L.ymref_init.argtypes = [C.POINTER(InitParams)]
        L.ymref_set_state.argtypes = [C.POINTER(C.c_void_p)]
        L.ymref_get_state.argtypes = [C.POINTER(C.c_void_p)]
        L.ymref_step.argtypes = [C.c_int]
        L.ymref_energy.argtypes = [C.POINTER(C.c_double)]
        L.ymref_time_steps.argtypes = [C.c_int, C.POINTER(C.c_float)]
        self.shape = None

    def _ck(self, rc, what):
        if rc:
            raise RuntimeError(f"{what}: {self.lib.ymref_last_error().decode()}")

    def create(self, grid, params, raise_zmean_smem: bool = True):
        self._ck(self.lib.ymref_create(C.byref(grid), C.byref(params), int(raise_zmean_smem)), "ymref_create")
        self.shape = (NSTATE, grid.nz, grid.nx)

    def init(self, ip):
        self._ck(self.lib.ymref_init(C.byref(ip)), "ymref_init")

    def set_state(self, state: np.ndarray):
        st = np.ascontiguousarray(state, dtype=np.float64)
        self._ck(self.lib.ymref_set_state(_ptrs(st)), "ymref_set_state")

    def get_state(self) -> np.ndarray:
        st = np.empty(self.shape, np.float64)
        self._ck(self.lib.ymref_get_state(_ptrs(st)), "ymref_get_state")
        return st

    def step(self, n: int = 1):
        self._ck(self.lib.ymref_step(int(n)), "ymref_step")

    def energy(self) -> float:
        e = C.c_double()
        self._ck(self.lib.ymref_energy(C.byref(e)), "ymref_energy")
        return e.value

    def time_steps(self, n: int) -> float:
        ms = C.c_float()
        self._ck(self.lib.ymref_time_steps(int(n), C.byref(ms)), "ymref_time_steps")
        return ms.value

    def destroy(self):
        self.lib.ymref_destroy()
