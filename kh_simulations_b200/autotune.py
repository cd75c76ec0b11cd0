"""Per grid-size-class launch-shape autotuner.

For a grid-size class (NZ and NX rounded to powers of two, band filter on or
off) it times the fused FCT kernel for each candidate strip width (the tile
shape: 32, 64 or 128 x-sweep positions per beam) and z-segment length (the
unit of work the persistent CTAs share out: each runs a contiguous block of
segments, a strip's part as one piece with one 3-row halo warm-up), then the
split FCT form, then the number of steps per captured CUDA graph, and keeps
the fastest.
Results are cached in a JSON table (``tuned.json`` beside this module, or
the path in ``KH_TUNING_FILE``) that ``KHRun(tune=True)`` consults.

The reference has no tuner: its launch shapes are fixed
(ymgpu2d/main_ym.cu:220-221, YM_FCT.cu:34-35, 60-63).
"""
from __future__ import annotations

import ctypes as C
import json
import math
import os
from pathlib import Path

from . import _lib

TABLE = Path(os.environ.get("KH_TUNING_FILE", Path(__file__).with_name("tuned.json")))


def size_class(nx: int, nz: int, filtered: bool) -> str:
    return f"nx{2 ** round(math.log2(max(nx, 1)))}_nz{2 ** round(math.log2(max(nz, 1)))}_{'f' if filtered else 'n'}"


def load_table() -> dict:
    try:
        return json.loads(TABLE.read_text())
    except (OSError, ValueError):
        return {}


def lookup(nx: int, nz: int, filtered: bool):
    return load_table().get(size_class(nx, nz, filtered))


def candidates(nx: int, nz: int):
    tbs = [tb for tb in (32, 64, 128) if nx >= tb - 6]
    segs = sorted({s for s in (1, 16, 32, 64, 128) if s <= max(16, nz)})
    return [(tb, s) for tb in tbs for s in segs]


def tune(run, reps: int = 3, graph_candidates=(2, 4, 8), save: bool = True) -> dict:
    """Time the candidates on `run` (a KHRun, state initialised) and record
    the best shape for its size class.

    Timing advances the state by many steps; the run's state is saved first
    and put back afterwards, so the run continues its own trajectory from
    where it was (same state, step count and energy reference)."""
    import torch

    lib = _lib.load()
    torch.cuda.synchronize(run.device)
    step_count = run.step_count
    try:
        saved = run.state.clone()
    except torch.OutOfMemoryError:
        saved = run.state.cpu()
    try:
        return _tune(run, lib, reps, graph_candidates, save)
    finally:
        torch.cuda.synchronize(run.device)
        run.set_state(saved)
        run.step_count = step_count
        torch.cuda.synchronize(run.device)


def _tune(run, lib, reps, graph_candidates, save) -> dict:
    import torch

    stream = torch.cuda.Stream(device=run.device)
    out = (C.c_float * 8)()
    best = None
    timings = {}
    def fct_ms():
        _lib.check(lib.ymkh_stage_times(run.ctx, 1, C.c_void_p(stream.cuda_stream), out, 8), "warm-up")
        _lib.check(lib.ymkh_stage_times(run.ctx, reps, C.c_void_p(stream.cuda_stream), out, 8), "stage times")
        return out[0] / reps

    _lib.check(lib.ymkh_set_fct_mode(run.ctx, _lib.FCT_FUSED), "ymkh_set_fct_mode")
    for tb, seg in candidates(run.d.nx, run.d.nz):
        _lib.check(lib.ymkh_set_fct_shape(run.ctx, tb, seg), "ymkh_set_fct_shape")
        ms = fct_ms()
        timings[f"{tb}x{seg}"] = ms
        if best is None or ms < best[0]:
            best = (ms, _lib.FCT_FUSED, tb, seg)
    _, _, tb, seg = best
    _lib.check(lib.ymkh_set_fct_shape(run.ctx, tb, seg), "ymkh_set_fct_shape")
    # the split form (x pass + z-streaming pass through a scratch copy)
    _lib.check(lib.ymkh_set_fct_mode(run.ctx, _lib.FCT_SPLIT), "ymkh_set_fct_mode")
    ms = fct_ms()
    timings["split"] = ms
    if ms < best[0]:
        best = (ms, _lib.FCT_SPLIT, tb, seg)
    mode = best[1]
    _lib.check(lib.ymkh_set_fct_mode(run.ctx, mode), "ymkh_set_fct_mode")
    gbest = None
    for g in graph_candidates:
        _lib.check(lib.ymkh_set_graph_steps(run.ctx, g), "ymkh_set_graph_steps")
        n = 4 * g
        run.step(n, stream)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        run.step(n, stream)
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / n
        if gbest is None or ms < gbest[0]:
            gbest = (ms, g)
    _lib.check(lib.ymkh_set_graph_steps(run.ctx, gbest[1]), "ymkh_set_graph_steps")
    entry = {"fct_mode": "split" if mode == _lib.FCT_SPLIT else "fused", "fct_strip": tb, "fct_segment": seg,
             "graph_steps": gbest[1], "fct_ms": best[0],
             "step_ms": gbest[0], "fct_candidates_ms": timings}
    if save:
        table = load_table()
        table[size_class(run.d.nx, run.d.nz, bool(run.d.bands))] = entry
        TABLE.write_text(json.dumps(table, indent=1, sort_keys=True))
    return entry


def apply(run) -> bool:
    """Apply a cached shape for the run's size class; False if none."""
    e = lookup(run.d.nx, run.d.nz, bool(run.d.bands))
    if not e:
        return False
    lib = _lib.load()
    _lib.check(lib.ymkh_set_fct_shape(run.ctx, int(e["fct_strip"]), int(e["fct_segment"])), "ymkh_set_fct_shape")
    mode = _lib.FCT_SPLIT if e.get("fct_mode") == "split" else _lib.FCT_FUSED
    _lib.check(lib.ymkh_set_fct_mode(run.ctx, mode), "ymkh_set_fct_mode")
    _lib.check(lib.ymkh_set_graph_steps(run.ctx, int(e["graph_steps"])), "ymkh_set_graph_steps")
    return True
