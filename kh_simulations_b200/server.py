"""``KHServer``: continuous batching of Kelvin–Helmholtz runs.

Requests (an .ini-level ``RunConfig`` plus a step count) arrive over time.
The server admits them in arrival order while their device footprint fits
the memory budget, keeps every admitted run's state resident in HBM, and
advances all admitted runs together through one ``KHBatch`` (one fused FCT
and one fused Maxwell launch per step over every run's tiles, captured as
CUDA graphs).  Between step chunks it retires finished runs (freeing their
memory), halts runs that break the reference's energy rule
(ymgpu2d/main_ym.cu:249, 467-474) and admits waiting requests: continuous
batching.  It reports p50/p99 run latency (arrival to completion) and the
aggregate cell-steps/s; ``serve_sequential`` runs the same requests one by
one through the plain single-run step for comparison.

The reference has no serving layer: campaigns run one ``ym_coupled``
process per configuration (ymgpu2d/scripts/*.sh).
"""
from __future__ import annotations

import math
import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np

from .config import RunConfig, derive

BYTES_PER_CELL_STATE = 2 * 24 * 8  # two 24-array FP64 buffers


def footprint(cfg: RunConfig) -> int:
    """Device bytes a run holds while resident: both state buffers, the
    band-filter twiddles and coefficient scratch of its filter engine,
    diagnostics (the allocations of include/ymkh.h's context)."""
    d = derive(cfg)
    cells = d.nx * d.nz
    fp = BYTES_PER_CELL_STATE * cells
    if d.bands:
        js = [2 * (hi - lo + 1) for lo, hi in d.bands]
        fp += sum(j * d.nz * 8 for j in js)  # FP64 twiddle matrices
        if cfg.filter_engine == "tf32x3":
            # TF32 hi/lo tile images: twiddles (both orientations) per band,
            # G and C^T of the 21 filtered arrays (x, z and j padded to 128)
            xpad = -(-d.nx // 128) * 128
            zpad = -(-d.nz // 128) * 128
            jpad = [-(-j // 128) * 128 for j in js]
            fp += sum(4 * jp * zpad * 4 for jp in jpad)
            fp += 2 * 21 * xpad * zpad * 4 + 2 * 21 * xpad * max(jpad) * 4
        else:
            fp += 21 * max(js) * d.nx * 8  # FP64 coefficients
    fp += 64 * 1024 + 16 * d.nx
    return fp


@dataclass
class KHRequest:
    rid: int
    cfg: RunConfig
    steps: int
    arrival: float = 0.0           # seconds after the server starts
    admitted: float = math.nan
    finished: float = math.nan
    status: str = "pending"        # pending | running | done | halted | rejected | cancelled | unfinished
    cancel_at: float = math.inf    # seconds after the server starts: withdrawn from then on
    energy: float = math.nan
    state: np.ndarray | None = None

    @property
    def cells(self) -> int:
        d = derive(self.cfg)
        return d.nx * d.nz

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


@dataclass
class ServeReport:
    requests: list
    makespan: float
    cell_steps: int
    p50: float
    p99: float
    mode: str
    extra: dict = field(default_factory=dict)

    @property
    def cell_steps_per_s(self) -> float:
        return self.cell_steps / self.makespan if self.makespan > 0 else 0.0

    def summary(self) -> dict:
        n_done = sum(r.status in ("done", "halted") for r in self.requests)
        return {"mode": self.mode, "requests": len(self.requests), "completed": n_done,
                "unfinished": sum(r.status == "unfinished" for r in self.requests),
                "halted": sum(r.status == "halted" for r in self.requests),
                "rejected": sum(r.status == "rejected" for r in self.requests),
                "cancelled": sum(r.status == "cancelled" for r in self.requests),
                "makespan_s": self.makespan, "cell_steps": self.cell_steps,
                "cell_steps_per_s": self.cell_steps_per_s, "p50_latency_s": self.p50, "p99_latency_s": self.p99,
                **self.extra}


def _censor(reqs, end: float) -> None:
    """Requests that had arrived by `end` but never ran to the end are
    "unfinished", their latency censored at `end`."""
    for r in reqs:
        if r.status in ("pending", "running") and r.arrival <= end:
            r.status, r.finished = "unfinished", end


def _percentiles(reqs) -> tuple:
    """p50 / p99 latency over completed requests and over unfinished ones at
    their censored latency (so, with any unfinished, lower bounds)."""
    lat = [r.latency for r in reqs if r.status in ("done", "halted", "unfinished")]
    if not lat:
        return math.nan, math.nan
    return float(np.percentile(lat, 50)), float(np.percentile(lat, 99))


class KHServer:
    """Continuous-batching server on one GPU.

    budget_bytes: device memory the resident runs may hold together.
    chunk: steps between admission/retirement decisions.
    keep_state: copy each finished run's final state to the host.
    large_cells: runs of at least this many cells fill the GPU on their own
        (one persistent FCT/Maxwell kernel over their tiles already occupies
        every SM, and the lone-run schedule of 128-wide strips in contiguous
        blocks is faster than a batch's): they are stepped one at a time in
        arrival order, in turns with the smaller runs, which advance
        together as one batch.  0 batches every run.
    """

    def __init__(self, budget_bytes: int, device="cuda", chunk: int = 100, graph_steps: int = 4,
                 keep_state: bool = False, check_energy: bool = True, clock=time.perf_counter,
                 large_cells: int = 1 << 20):
        self.budget = int(budget_bytes)
        self.device = device
        self.chunk = int(chunk)
        self.graph_steps = graph_steps
        self.keep_state = keep_state
        self.check_energy = check_energy
        self.clock = clock
        self.large_cells = int(large_cells)

    # ---------------------------------------------------------------- helpers
    def _start_run(self, req: KHRequest, stream=None, must: bool = True):
        """A new run for `req`, initialised on `stream`.  If the device has
        no room for it (the budget counts live runs, but the caching
        allocator may still hold pieces of retired ones), cached memory is
        released and the creation retried once; if that fails too, None is
        returned when `must` is false (the caller retries after retiring
        runs), else the error is raised."""
        import torch

        from ._lib import YMKHError
        from .run import KHRun

        def create():
            try:
                return KHRun(req.cfg, device=self.device, graph_steps=self.graph_steps)
            except (YMKHError, torch.OutOfMemoryError):
                if must and attempt == 1:
                    raise
                return None

        run = None
        for attempt in (0, 1):
            run = create()
            if run is not None:
                break
            torch.cuda.synchronize(self.device)
            torch.cuda.empty_cache()
        if run is None:
            return None
        run.init(stream=stream)
        run.E0 = run.energy(stream)
        return run

    def _finish(self, req: KHRequest, run, status: str, t: float):
        req.finished = t
        req.status = status
        if self.keep_state:
            req.state = run.state_numpy()
        req.energy = run.energy()
        run.close()

    def admit_order(self, pending: deque, now: float, used: int) -> list:
        """FIFO admission by footprint: admit the arrived head while it fits;
        a request larger than the whole budget is rejected."""
        out = []
        while pending and pending[0].arrival <= now:
            req = pending[0]
            fp = footprint(req.cfg)
            if fp > self.budget:
                pending.popleft()
                req.status = "rejected"
                continue
            if used + fp > self.budget:
                break
            pending.popleft()
            used += fp
            out.append((req, fp))
        return out

    def _halted_many(self, runs, stream) -> list:
        """The reference's halt rule for several runs, with their energies
        reduced on the device and read back by one synchronisation (the
        error words of the batch's kernels are checked by the caller)."""
        import ctypes as C

        import torch

        if not self.check_energy or not runs:
            return [False] * len(runs)
        out = torch.empty(len(runs), dtype=torch.float64, device=runs[0].device)
        lib = runs[0].lib
        for i, run in enumerate(runs):
            rc = lib.ymkh_energy_async(run.ctx, C.c_void_p(out.data_ptr() + 8 * i), C.c_void_p(stream.cuda_stream))
            if rc:
                from ._lib import check

                check(rc, "ymkh_energy_async")
        stream.synchronize()
        es = out.cpu().tolist()
        return [not math.isfinite(e) or e / r.E0 > r.d.energy_thresh for e, r in zip(es, runs)]

    def _halted(self, run, stream) -> bool:
        if not self.check_energy:
            return False
        e = run.energy(stream)
        return not math.isfinite(e) or e / run.E0 > run.d.energy_thresh

    # ------------------------------------------------------------------ serve
    def serve(self, requests: list, deadline: float = math.inf) -> ServeReport:
        """Serve `requests` (arrival times in seconds after the start).

        Small runs (below large_cells) join one KHBatch as they are admitted
        and leave it when done; large runs wait resident in HBM and the
        oldest is stepped alone.  Each round enqueues up to `chunk` steps of
        the batch and then up to `chunk` steps of the oldest large run;
        while they run, arrived requests are admitted and initialised
        on a separate stream; finished and halted runs retire between
        rounds.  With a finite `deadline` (seconds after the start) the
        server stops there: unfinished runs count the steps they made and
        are reported as "unfinished" (their latency is censored at the
        deadline)."""
        import torch

        from .batch import KHBatch

        # the batch and the oldest large run share one stream and take turns:
        # a large run's persistent kernels give each CTA one contiguous block
        # of work, so kernels of another stream holding some SMs would delay
        # the whole launch
        s_run = torch.cuda.Stream(device=self.device)
        s_small = s_large = s_run
        s_admit = torch.cuda.Stream(device=self.device)
        batch = KHBatch(device=self.device, graph_steps=self.graph_steps)
        pending = deque(sorted(requests, key=lambda r: (r.arrival, r.rid)))
        small: list = []   # [req, run, fp, remaining]
        large: deque = deque()
        used = 0
        cell_steps = 0
        t0 = self.clock()
        self.deferred = 0
        first = pending[0].arrival if pending else 0.0
        while pending or small or large:
            now = self.clock() - t0
            if now >= deadline:
                break
            for req in [r for r in pending if r.cancel_at <= now]:  # withdrawn before admission
                pending.remove(req)
                req.status, req.finished = "cancelled", now
            # this round's work on the resident runs
            ks = min(self.chunk, min(a[3] for a in small)) if small else 0
            kl, head = 0, None
            if large:
                head = large[0]
                kl = min(self.chunk, head[3])
            if ks:
                batch.step(ks, s_small)
            if kl:
                head[1].step(kl, s_large)
            # admissions while the device works; new runs start on their own stream
            admitted = []
            cand = self.admit_order(pending, now, used)
            for i, (req, fp) in enumerate(cand):
                # with runs resident, a creation that finds no room waits,
                # with the candidates after it, at the head of the queue for
                # runs to retire
                run = self._start_run(req, s_admit, must=not (small or large or admitted))
                if run is None:
                    for r, _ in reversed(cand[i:]):
                        pending.appendleft(r)
                    self.deferred += 1
                    break
                req.admitted = self.clock() - t0
                req.status = "running"
                admitted.append([req, run, fp, req.steps])
                used += fp
            if not ks and not kl and not admitted:
                if pending:
                    time.sleep(max(0.0, min(0.05, pending[0].arrival - (self.clock() - t0))))
                continue
            s_run.synchronize()
            for a in small:
                a[3] -= ks
                cell_steps += ks * a[0].cells
            if kl:
                head[3] -= kl
                cell_steps += kl * head[0].cells
            t = self.clock() - t0
            done, keep = [], []
            if ks:
                batch.check(s_small)  # bounded in-kernel waits of the batch's step
            halts = self._halted_many([a[1] for a in small], s_small) if ks else [False] * len(small)
            for a, h in zip(small, halts):
                req, run, fp, rem = a
                status = ("done" if rem <= 0 else "cancelled" if req.cancel_at <= t
                          else "halted" if h else None)
                if status:
                    batch.remove(run)
                    done.append((a, status))
                else:
                    keep.append(a)
            small = keep
            if kl:
                req, run, fp, rem = head
                status = ("done" if rem <= 0 else "cancelled" if req.cancel_at <= t
                          else "halted" if self._halted(run, s_large) else None)
                if status:
                    large.popleft()
                    done.append((head, status))
            for a in [a for a in large if a[0].cancel_at <= t]:  # withdrawn while waiting
                large.remove(a)
                done.append((a, "cancelled"))
            for (req, run, fp, _), status in done:
                self._finish(req, run, status, self.clock() - t0)
                used -= fp
            for a in admitted:
                if self.large_cells > 0 and a[0].cells >= self.large_cells:
                    large.append(a)
                else:
                    batch.add(a[1])
                    small.append(a)
        end = self.clock() - t0
        for req, run, fp, rem in small + list(large):
            req.status, req.finished = "unfinished", end
            run.close()
        _censor(requests, end)
        batch.close()
        makespan = end - first
        p50, p99 = _percentiles(requests)
        return ServeReport(requests, makespan, cell_steps, p50, p99, "batched",
                           {"large_cells": self.large_cells, "deferred_admissions": self.deferred,
                            "unfinished": sum(r.status == "unfinished" for r in requests)})

    def serve_sequential(self, requests: list, deadline: float = math.inf) -> ServeReport:
        """The same requests one by one through the plain single-run step, in
        arrival order (a request starts when it has arrived and the previous
        one has finished).  `deadline` as in serve()."""
        import torch

        stream = torch.cuda.Stream(device=self.device)
        order = sorted(requests, key=lambda r: (r.arrival, r.rid))
        t0 = self.clock()
        first = order[0].arrival if order else 0.0
        cell_steps = 0
        for req in order:
            if self.clock() - t0 >= deadline:
                break
            if footprint(req.cfg) > self.budget:
                req.status = "rejected"
                continue
            if req.cancel_at <= self.clock() - t0:
                req.status, req.finished = "cancelled", self.clock() - t0
                continue
            now = self.clock() - t0
            if req.arrival > now:
                if req.arrival >= deadline:
                    break
                time.sleep(req.arrival - now)
            run = self._start_run(req, stream)
            req.admitted = self.clock() - t0
            status = "done"
            left = req.steps
            while left > 0:
                if req.cancel_at <= self.clock() - t0:
                    status = "cancelled"
                    break
                if self.clock() - t0 >= deadline:
                    status = "unfinished"
                    break
                k = min(self.chunk, left)
                run.step(k, stream)
                left -= k
                cell_steps += k * req.cells
                if self._halted(run, stream):
                    status = "halted"
                    break
            stream.synchronize()
            if status == "unfinished":
                req.status, req.finished = status, self.clock() - t0
                run.close()
            else:
                self._finish(req, run, status, self.clock() - t0)
        end = self.clock() - t0
        _censor(order, end)
        makespan = end - first
        p50, p99 = _percentiles(order)
        return ServeReport(order, makespan, cell_steps, p50, p99, "sequential",
                           {"unfinished": sum(r.status == "unfinished" for r in order)})


def poisson_mix(seed: int, rate: float, duration: float, min_cells: int, max_cells: int, min_steps: int,
                max_steps: int, base_ini: str, nz_multiple: int = 32, keep_third: bool = False,
                filter_engine: str = "dft") -> list:
    """Seeded request mix: Poisson arrivals at `rate` per second for
    `duration` seconds; cell counts log-uniform in [min_cells, max_cells]
    with NZ:NX = 1:2 (NZ rounded to a multiple of nz_multiple, a power of two
    when the run suppresses kz=0); V0 ~ U[0.02, 0.2], shear width
    ~ U[0.5, 2], kz in {0..3}, perturbation ~ U[0.05, 0.2]; kz = 0 suppressed
    in every other request; steps uniform in [min_steps, max_steps].  With
    keep_third, every request filters modes above NZ/3 with the given
    filter engine."""
    from .config import loads

    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    rid = 0
    while True:
        t += rng.exponential(1.0 / rate)
        if t > duration:
            break
        cells = math.exp(rng.uniform(math.log(min_cells), math.log(max_cells)))
        kz0 = rid % 2 == 0
        nz = math.sqrt(cells / 2.0)
        if kz0:
            nz = 2 ** int(round(math.log2(nz)))
        else:
            nz = max(nz_multiple, int(round(nz / nz_multiple)) * nz_multiple)
        nx = 2 * nz
        v0 = rng.uniform(0.02, 0.2)
        eps = rng.uniform(0.5, 2.0)
        kz = int(rng.integers(0, 4))
        amp = rng.uniform(0.05, 0.2)
        steps = int(rng.integers(min_steps, max_steps + 1))
        dz = 2 * math.pi / nz
        dx = 20.0 / nx
        # CFL-safe Courant number: dt * sqrt(dx^-2 + dz^-2) <= 0.4 with dt = C dx
        courant = min(0.4, 0.4 / (dx * math.sqrt(dx ** -2 + dz ** -2)))
        ini = (base_ini + f"k_mode = {kz}\nV0 = {v0:.6f}\neps_override = {eps:.6f}\nperturb_amp = {amp:.6f}\n"
               f"nz_override = {nz}\nnx_override = {nx}\ncourant_override = {courant:.6f}\n"
               f"suppress_kz0 = {1 if kz0 else 0}\n")
        if keep_third:
            ini += f"kz_keep_max = {nz // 3}\nfilter_engine = {filter_engine}\n"
        out.append(KHRequest(rid, loads(ini, f"req{rid}"), steps, t))
        rid += 1
    return out


def cfl_courant(nx: int, nz: int, lx: float = 20.0, lz: float = 2 * math.pi, target: float = 0.4) -> float:
    """Courant number C (dt = C dx) with dt * sqrt(dx^-2 + dz^-2) <= target,
    capped at `target`."""
    dx, dz = lx / nx, lz / nz
    return min(target, target / (dx * math.sqrt(dx ** -2 + dz ** -2)))


def uneven_sweep(seed: int, n: int, base_ini: str = "") -> list:
    """Seeded uneven-size sweep of n runs: NZ in {128, 256, 512, 1024} and
    NX in {256, 512, 1024, 2048} drawn uniformly, V0 ~ U[0.02, 0.2], shear
    width ~ U[0.5, 2], kz in {0..3}, perturbation ~ U[0.05, 0.2], kz = 0
    suppressed in the runs of even index, CFL-safe Courant number.
    Returns RunConfigs."""
    from .config import loads

    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        nz = int(rng.choice([128, 256, 512, 1024]))
        nx = int(rng.choice([256, 512, 1024, 2048]))
        v0 = rng.uniform(0.02, 0.2)
        eps = rng.uniform(0.5, 2.0)
        kz = int(rng.integers(0, 4))
        amp = rng.uniform(0.05, 0.2)
        ini = (base_ini + f"k_mode = {kz}\nV0 = {v0:.6f}\neps_override = {eps:.6f}\nperturb_amp = {amp:.6f}\n"
               f"nz_override = {nz}\nnx_override = {nx}\ncourant_override = {cfl_courant(nx, nz):.6f}\n"
               f"suppress_kz0 = {1 if i % 2 == 0 else 0}\n")
        out.append(loads(ini, f"sweep{i}"))
    return out


def split_precision_runs(seed: int, n: int, base_ini: str = "", nz: int = 1024, nx: int = 2048) -> list:
    """n runs at NZ x NX with the uneven sweep's parameter ranges (seed `seed`)
    and the band filter keeping |k| <= NZ/3."""
    from .config import loads

    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        v0 = rng.uniform(0.02, 0.2)
        eps = rng.uniform(0.5, 2.0)
        kz = int(rng.integers(0, 4))
        amp = rng.uniform(0.05, 0.2)
        ini = (base_ini + f"k_mode = {kz}\nV0 = {v0:.6f}\neps_override = {eps:.6f}\nperturb_amp = {amp:.6f}\n"
               f"nz_override = {nz}\nnx_override = {nx}\ncourant_override = {cfl_courant(nx, nz):.6f}\n"
               f"suppress_kz0 = {1 if i % 2 == 0 else 0}\nkz_keep_max = {nz // 3}\n")
        out.append(loads(ini, f"split{i}"))
    return out

