"""``KHBatch``: many runs of any grid size advancing together.

Each batch step launches one fused FCT kernel and one fused Maxwell kernel
over the flattened (run, strip, segment) work list of every member, then
the per-run filter stages (include/ymkh.h, ymkh_batch_*).  A run's state
after k batch steps is bit-identical to k steps of the run alone.
Membership may change between calls: that is what the serving loop uses
for continuous batching.
"""
from __future__ import annotations

import ctypes as C

import torch

from . import _lib
from ._lib import check
from .run import KHRun, _stream_ptr


class KHBatch:
    def __init__(self, device="cuda", graph_steps: int | None = None):
        self.lib = _lib.load()
        self.device = torch.device(device)
        h = C.c_void_p()
        with torch.cuda.device(self.device):
            check(self.lib.ymkh_batch_create(C.byref(h)), "ymkh_batch_create")
        self.h = h
        if graph_steps is not None:
            check(self.lib.ymkh_batch_set_graph_steps(self.h, graph_steps), "ymkh_batch_set_graph_steps")
        self.runs: list[KHRun] = []

    def add(self, run: KHRun) -> None:
        check(self.lib.ymkh_batch_add(self.h, run.ctx), "ymkh_batch_add")
        self.runs.append(run)

    def remove(self, run: KHRun) -> None:
        check(self.lib.ymkh_batch_remove(self.h, run.ctx), "ymkh_batch_remove")
        self.runs.remove(run)

    def __len__(self) -> int:
        return len(self.runs)

    def step(self, n: int = 1, stream=None) -> None:
        if not self.runs or n <= 0:
            return
        with torch.cuda.device(self.device):
            check(self.lib.ymkh_batch_step(self.h, int(n), C.c_void_p(_stream_ptr(stream))), "ymkh_batch_step")
        for r in self.runs:
            r.step_count += n

    def check(self, stream=None) -> None:
        check(self.lib.ymkh_batch_check(self.h, C.c_void_p(_stream_ptr(stream))), "ymkh_batch_check")

    def cells(self) -> int:
        return sum(r.d.nx * r.d.nz for r in self.runs)

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.ymkh_batch_destroy(self.h)
            self.h = None

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass
