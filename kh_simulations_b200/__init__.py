"""B200-native Kelvin–Helmholtz step of the 2D two-fluid SU(2) Yang–Mills
simulator (drop-in for the step loop of ymgpu2d/main_ym.cu).

The arithmetic runs in the in-tree CUDA library ``libymkh.so`` (C ABI in
include/ymkh.h, built by ``python -m kh_simulations_b200.build``); this
package holds the configuration layer, the run and batch drivers and the
serving loop.  Importing it does not need a GPU; running does.
"""
from .config import RunConfig, derive, load_config, loads  # noqa: F401

__all__ = ["RunConfig", "derive", "load_config", "loads", "KHRun", "KHBatch", "KHServer"]


def __getattr__(name):
    if name == "KHRun":
        from .run import KHRun

        return KHRun
    if name == "KHBatch":
        from .batch import KHBatch

        return KHBatch
    if name == "KHServer":
        from .server import KHServer

        return KHServer
    raise AttributeError(name)
