#!/usr/bin/env python
"""Throughput of the Kelvin–Helmholtz step (cell-steps/s) on B200.

Workload (default): the plain single large run, 4096 x 8192 — NZ = 4096
cells along the periodic flow axis (Lz = 2 pi) by NX = 8192 along the shear
axis (Lx = 20) — FP64, V0 = 0.05, shear width 1, kz = 1 seed of amplitude
0.15 V0 on Az2/Az3 (run_mode 6), alpha = 1, CFL 0.4.  Synthetic: the
initial state is the reference's analytic equilibrium plus seed.

Filter: the reference's band-filter kernels launch one thread per z cell
and cannot launch for NZ > 1024 (ymgpu2d/main_ym.cu:396, YM_Physics.cu:349),
so the reference's own step at this size performs no filtering; the default
``--filter ref`` reproduces that.  ``--filter keep`` subtracts modes above
NZ/3 every step with the dense FP64 contraction; the ``filter_keep``
field times config 1 as stated (filter on) with both filter engines.

One step = one iteration of the reference loop over the whole grid.  The
state (12.9 GB for two buffers) is far larger than L2 (126 MB), so no flush
is needed between steps.  N > 1: independent replicas, one per GPU (the
path does not shard across GPUs), ``scaling: weak``.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))
# The served leg creates and frees about a thousand runs of mixed sizes; with
# expandable segments torch's caching allocator maps device memory in pages
# and can return freed pages, so pieces of retired runs' buffers do not keep
# whole segments reserved (set before torch first touches the device).
os.environ.setdefault("PYTORCH_CUDA_ALLOC_CONF", "expandable_segments:True")

WORKLOADS = {
    # name: (NX shear, NZ periodic)
    "kh_4096x8192": (8192, 4096),
    "kh_256x512": (512, 256),
    # profiling size: 805 MB per state buffer (> L2), for ncu captures
    "kh_1024x2048": (2048, 1024),
}
PHYSICS = ("k_mode = 1\nalpha_YM = 1.0\nperturb_amp = 0.15\nrun_mode = 6\nV0 = 0.05\neps_override = 1.0\n"
           "lx_override = 20\ncourant_override = 0.4\n")
BYTES_STEP = 376  # compulsory: read 24 FP64 arrays, write 23 (Az1 frozen)
L2_BYTES = 126 << 20  # B200 L2
BYTES_FCT = 288   # fct_fused_kernel: read 12 fluid + 12 field arrays, write 12 fluid
BYTES_MAXWELL = 280  # maxwell_fused_kernel: read 24, write 11 (Az1 frozen)


def ini_for(workload: str, filt: str, engine: str = "dft") -> str:
    nx, nz = WORKLOADS[workload]
    text = PHYSICS + f"nx_override = {nx}\nnz_override = {nz}\nfilter_engine = {engine}\n"
    if filt == "keep" or (filt == "ref" and nz <= 1024):
        text += f"kz_keep_max = {nz // 3}\n"
    return text


def measured_peaks() -> tuple:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.lines: list[str] = []
        self.proc = None
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.idx)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_oracle_rate(workload: str, steps: int, threads: int | None = None, min_seconds: float = 0.0) -> dict:
    """The FP64 OpenMP oracle on a bounded sample of the workload: the full
    shear extent and NZ reduced to 256 rows (the step's per-cell work does not
    depend on NZ when no band filter runs).  Runs `steps` steps, then more
    one at a time until `min_seconds` of work have been timed."""
    import numpy as np

    from kh_simulations_b200._lib import Grid
    from kh_simulations_b200.config import derive, loads, step_params
    from oracle import Oracle

    if threads:
        os.environ["OMP_NUM_THREADS"] = str(threads)
    nx, _ = WORKLOADS[workload]
    nz = 256
    cfg = loads(PHYSICS + f"nx_override = {nx}\nnz_override = {nz}\n")
    d = derive(cfg)
    g = Grid(d.nx, d.nz, d.dx, d.dz)
    p = step_params(cfg, d)
    orc = Oracle()
    st = np.zeros((24, nz, nx))
    st[12] = st[18] = 1.0
    st[15], st[21] = 1.0, -1.0
    x = np.arange(nx)
    xi = (x * d.dx - nx * d.dx * 0.5) / d.eps
    st[14] = d.V0 * np.tanh(xi)[None, :]
    st[20] = -st[14]
    orc.step(g, p, st, 1)  # warm-up (page-in, thread pool)
    t0 = time.perf_counter()
    orc.step(g, p, st, steps)
    dt = time.perf_counter() - t0
    while dt < min_seconds:
        orc.step(g, p, st, 1)
        steps += 1
        dt = time.perf_counter() - t0
    return {"value": nx * nz * steps / dt, "unit": "cell-steps/s", "cores": orc.threads(), "kind": "port",
            "sample": f"FP64 OpenMP oracle, {steps} step(s) of the same physics on {nz}x{nx} (NZ x NX) = "
                      f"{nx * nz} cells, no band filter, {dt:.2f} s"}


CONFIG0 = PHYSICS + "nz_override = 256\nnx_override = 512\nkz_keep_max = 85\n"


def cpu_baselines(repeats: int = 5) -> dict:
    """The FP64 OpenMP oracle on all host cores, median of `repeats` timed
    runs each: config 0 (256 x 512, keep |k| <= 85, the band filter with the
    FP32 twiddle table) for 5 steps, and the first 8 runs of the uneven sweep
    (seed 1, config 2's distributions) for 1 step each, as an aggregate."""
    import numpy as np

    from kh_simulations_b200._lib import Grid
    from kh_simulations_b200.config import derive, loads, step_params
    from kh_simulations_b200.server import uneven_sweep
    from oracle import Oracle

    orc = Oracle()

    def initial(d):
        st = np.zeros((24, d.nz, d.nx))
        st[12] = st[18] = 1.0
        st[15], st[21] = 1.0, -1.0
        xi = (np.arange(d.nx) * d.dx - d.nx * d.dx * 0.5) / d.eps
        st[14] = d.V0 * np.tanh(xi)[None, :]
        st[20] = -st[14]
        st[10] = 1e-3 * np.cos(2 * np.pi * np.arange(d.nz) / d.nz)[:, None]
        return st

    def setup(cfg):
        d = derive(cfg)
        tw = None
        if d.bands:
            tw = orc.twiddles(d.nz, 0, max(hi for _, hi in d.bands))
        return d, Grid(d.nx, d.nz, d.dx, d.dz), step_params(cfg, d), initial(d), tw

    out = {"cores": orc.threads(), "kind": "port", "repeats": repeats, "statistic": "median"}
    d, g, p, st, tw = setup(loads(CONFIG0))
    orc.step(g, p, st, 1, twiddles=tw)
    rates = []
    for _ in range(repeats):
        t0 = time.perf_counter()
        orc.step(g, p, st, 5, twiddles=tw)
        rates.append(d.nx * d.nz * 5 / (time.perf_counter() - t0))
    out["config0"] = {"value": statistics.median(rates), "unit": "cell-steps/s",
                      "sample": "256x512 (NZ x NX), keep |k| <= 85 (band filter on), 5 steps per run"}
    runs = [setup(c) for c in uneven_sweep(1, 8, SWEEP_BASE)]
    for d, g, p, st, tw in runs:
        orc.step(g, p, st, 1, twiddles=tw)
    rates = []
    for _ in range(repeats):
        t0 = time.perf_counter()
        for d, g, p, st, tw in runs:
            orc.step(g, p, st, 1, twiddles=tw)
        rates.append(sum(d.nx * d.nz for d, *_ in runs) / (time.perf_counter() - t0))
    out["config2_subset"] = {"value": statistics.median(rates), "unit": "cell-steps/s",
                             "sample": "first 8 runs of the uneven sweep (seed 1), 1 step each, aggregate"}
    return out


def run_reference(args, world, rank, local):
    """Reference arm: the reference's own step on the host cores (it has no
    CPU implementation, so this is the FP64 OpenMP port), plus the
    reference's own CUDA kernels timed on this GPU when the harness is built."""
    if rank != 0:
        return 0
    per = []
    cb = None
    for k in range(args.warmup + args.steps):
        r = cpu_oracle_rate(args.workload, 1)
        if k >= args.warmup:
            per.append(r["value"])
            cb = r
    value = statistics.median(per)
    line = {"metric": "cell-steps/s", "value": value, "unit": "cell-steps/s", "impl": "reference",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": args.workload,
                       "filter": ("keep |k| <= NZ/3" if WORKLOADS[args.workload][1] <= 1024
                                  else "none (reference cannot launch its band filter for NZ > 1024)")},
            "cpu_baseline": {**cb, "value": value},
            "e2e": {"value": value, "unit": "cell-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    try:
        line["reference_cuda"] = ref_cuda_rate(args)
        line["reference_cuda_config0"] = ref_cuda_rate(args, CONFIG0, steps=200,
                                                       what="config 0: 256x512, keep |k| <= 85")
        if args.ref_sweep_runs > 0:
            line["reference_cuda_sweep"] = ref_sweep_rate(args, args.ref_sweep_runs)
    except Exception as e:  # the CPU arm stands on its own
        line["reference_cuda"] = {"unavailable": str(e)[:200]}
    if not args.no_cpu_baseline:
        line["cpu_baselines"] = cpu_baselines()
    print(json.dumps(line), flush=True)
    return 0


def ref_cuda_rate(args, ini: str | None = None, steps: int | None = None, what: str | None = None) -> dict:
    """The reference's own kernels (oracle/_ref/libymref.so, its stock
    flags) through its own stage sequence, timed with CUDA events, on the
    workload (or on `ini`)."""
    import torch

    from kh_simulations_b200._lib import Grid
    from kh_simulations_b200.config import derive, loads, step_params
    from kh_simulations_b200.run import init_params
    from oracle import REF_STOCK_LIB, RefHarness

    if not torch.cuda.is_available() or not REF_STOCK_LIB.exists():
        raise RuntimeError("no GPU or reference harness not built")
    cfg = loads(ini if ini else ini_for(args.workload, "ref"))
    steps = steps or args.steps
    d = derive(cfg)
    ref = RefHarness(parity=False)
    ref.create(Grid(d.nx, d.nz, d.dx, d.dz), step_params(cfg, d))
    ip, _k = init_params(cfg, d)
    ref.init(ip)
    ref.step(max(1, args.warmup))
    ms = ref.time_steps(steps)
    ref.destroy()
    cells = d.nx * d.nz
    out = {"value": cells * steps / (ms / 1e3), "unit": "cell-steps/s", "ms_per_step": ms / steps,
           "build": "reference sources unmodified, nvcc -O2 sm_100a (its stock flags)"}
    if what:
        out["workload"] = what
    return out


def ref_sweep_rate(args, nruns: int) -> dict:
    """The reference's own kernels (stock build) over the uneven sweep of
    the batched leg (seed 1, `nruns` runs), one run after another as its
    campaign scripts run them: aggregate cell-steps/s over the timed steps."""
    from kh_simulations_b200._lib import Grid
    from kh_simulations_b200.config import derive, step_params
    from kh_simulations_b200.run import init_params
    from kh_simulations_b200.server import uneven_sweep
    from oracle import REF_STOCK_LIB, RefHarness

    if not REF_STOCK_LIB.exists():
        raise RuntimeError("reference harness not built")
    ms_total, cell_steps = 0.0, 0
    for cfg in uneven_sweep(1, nruns, SWEEP_BASE):
        d = derive(cfg)
        ref = RefHarness(parity=False)
        ref.create(Grid(d.nx, d.nz, d.dx, d.dz), step_params(cfg, d))
        ip, _k = init_params(cfg, d)
        ref.init(ip)
        ref.step(max(1, args.warmup))
        ms_total += ref.time_steps(args.steps)
        cell_steps += d.nx * d.nz * args.steps
        ref.destroy()
    return {"workload": f"uneven sweep, {nruns} runs (seed 1), {args.steps} steps each, one run after another",
            "value": cell_steps / (ms_total / 1e3), "unit": "cell-steps/s"}


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=4)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="kh_4096x8192")
    ap.add_argument("--filter", choices=["ref", "keep"], default="ref")
    ap.add_argument("--filter-engine", choices=["dft", "tf32x3"], default="dft",
                    help="band filter of the main run: FP64 sums or 3-pass TF32 on the tensor cores")
    ap.add_argument("--no-config0", action="store_true", help="skip the config-0 leg (256 x 512, keep |k| <= 85)")
    ap.add_argument("--no-filter-keep", action="store_true",
                    help="skip the config-1-as-stated leg (filter on at the workload size, both engines)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-filter-leg", action="store_true", help="skip the FP64 vs TF32 band filter leg")
    ap.add_argument("--filter-error-steps", type=int, default=0, help="steps of the TF32-vs-FP64 filter error leg")
    ap.add_argument("--filter-error-runs", type=int, default=2)
    ap.add_argument("--filter-error-control", action="store_true",
                    help="the error leg as a control: FP64 filter against FP64 filter with nA scaled by 1+2^-52 at the start")
    ap.add_argument("--batched-runs", type=int, default=64, help="runs in the batched-vs-plain leg (0: skip)")
    ap.add_argument("--batched-steps", type=int, default=2000, help="steps per run in the batched-vs-plain leg")
    ap.add_argument("--ref-sweep-runs", type=int, default=64,
                    help="--impl reference: also time the reference's kernels over the uneven sweep (0: skip)")
    ap.add_argument("--batch-by-size", action="store_true",
                    help="opt-in leg: batched against plain for identical runs of each size, 128x256 .. 1024x2048")
    ap.add_argument("--served-seconds", type=float, default=60.0, help="arrival window of the served leg (0: skip)")
    ap.add_argument("--served-drain", type=float, default=60.0,
                    help="served leg: each pass stops this long after the last arrival at the latest "
                         "(a safety bound; the default mix drains well before it)")
    ap.add_argument("--served-step-scale", type=int, default=200,
                    help="served leg: config 4's 2000..20000 steps per request divided by this")
    ap.add_argument("--served-fp64-seconds", type=float, default=6.0,
                    help="arrival window of the served leg with the FP64 filter (0: skip)")
    ap.add_argument("--served-check", type=int, default=6,
                    help="requests in the served tolerance check against plain FP64 runs (0: skip)")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)

    from kh_simulations_b200 import replicas

    if args.impl == "reference":
        # rank 0 alone times the reference on the host cores; other ranks
        # exit at once (no process group: the arm has no collective)
        world = int(os.environ.get("WORLD_SIZE", "1"))
        rank = int(os.environ.get("RANK", "0"))
        return run_reference(args, world, rank, int(os.environ.get("LOCAL_RANK", "0")))
    rk = replicas.init("nccl")
    world, rank, local = rk.world, rk.rank, rk.local

    import torch

    from kh_simulations_b200 import _lib
    from kh_simulations_b200.config import loads
    from kh_simulations_b200.run import KHRun

    dev = torch.device(f"cuda:{local}")
    torch.cuda.set_device(dev)
    cfg = loads(ini_for(args.workload, args.filter, args.filter_engine))
    run = KHRun(cfg, device=dev)
    run.init()
    d = run.d
    cells = d.nx * d.nz
    stream = torch.cuda.Stream(device=dev)
    run.step(args.warmup, stream)
    torch.cuda.synchronize(dev)
    replicas.barrier(rk)

    sampler = ClockSampler(dev.index if dev.index is not None else 0)
    sampler.start()
    time.sleep(0.3)
    l0 = _lib.launch_count()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(dev)
    e0.record(stream)
    run.step(args.steps, stream)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    launches = _lib.launch_count() - l0
    clocks = sampler.stop()
    ms = e0.elapsed_time(e1)
    ms_max = replicas.max_over_ranks(ms, rk)
    replicas.barrier(rk)
    value = replicas.aggregate_rate(cells * args.steps, ms_max, rk)

    # per-stage device times (separate uncaptured pass, events between stages)
    nst = 3
    out = (C.c_float * 8)()
    _lib.check(_lib.load().ymkh_stage_times(run.ctx, nst, C.c_void_p(stream.cuda_stream), out, 8), "stage times")
    stage_ms = {n: out[i] / nst for i, n in enumerate(_lib.STAGES)}
    dom = max(stage_ms, key=stage_ms.get)
    peak, peak_kind = measured_peaks()
    alg = {"fct": BYTES_FCT, "maxwell": BYTES_MAXWELL}.get(dom)
    roof = None
    if alg is not None:
        achieved = alg * cells / (stage_ms[dom] / 1e3) / 1e9
        traffic = None
        tf = ROOT / "profiles" / "traffic.json"
        if tf.exists():
            t = json.loads(tf.read_text()).get(dom)
            if t:
                traffic = t * cells
        roof = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": traffic, "peak_source": peak_kind,
                "algorithmic_bytes_per_cell": alg}
    step_gbs = BYTES_STEP * cells / (ms / args.steps / 1e3) / 1e9

    line = {"metric": "cell-steps/s", "value": value, "unit": "cell-steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": args.workload, "nz_periodic": d.nz, "nx_shear": d.nx,
                       "filter": "keep |k| <= NZ/3" if d.bands else "none (as the reference at NZ > 1024)",
                       "l2": (f"state {2 * 24 * 8 * cells / 1e9:.2f} GB > L2 (126 MB); no flush needed"
                              if 2 * 24 * 8 * cells > L2_BYTES else
                              f"state {2 * 24 * 8 * cells / 1e6:.0f} MB fits in L2 (126 MB): L2-resident, "
                              "not a roofline workload"),
                       "parallelism": f"replicas x{world}",
                       "graph_steps": 4},
            "roofline": roof,
            "step_roofline": {"bytes_per_cell_step": BYTES_STEP, "achieved": step_gbs, "peak": peak,
                              "frac": step_gbs / peak, "unit": "GB/s"},
            "stage_ms": stage_ms, "clocks": clocks, "gpu_launches": launches}

    if not args.no_e2e:
        line["e2e"] = e2e_rate(run, args, stream, rk)
    run.close()
    del run
    torch.cuda.empty_cache()

    if world == 1 and not args.no_filter_keep and args.filter == "ref" and d.nz > 1024:
        line["filter_keep"] = filter_keep_rate(args, dev)
    if world == 1 and not args.no_filter_leg:
        line["filter"] = filter_engines(args, dev)
    if world == 1 and args.filter_error_steps > 0:
        line["filter_error"] = filter_error(args, dev, args.filter_error_steps, args.filter_error_runs,
                                            control=args.filter_error_control)
    if world == 1 and args.batched_runs > 0:
        line["batched"] = batched_rate(args, dev, args.batched_runs, args.batched_steps)
    if world == 1 and args.batch_by_size:
        line["batch_by_size"] = batch_by_size(dev)
    if world == 1 and args.served_seconds > 0:
        line["served"] = served_rate(args, dev, args.served_seconds)
    if world == 1 and not args.no_config0:
        line["config0"] = config0_rate(dev)
    if world == 1 and not args.no_cpu_baseline:  # a host-core figure, taken at N = 1 only
        line["cpu_baseline"] = cpu_oracle_rate(args.workload, 1, min_seconds=10.0)
        line["cpu_baselines"] = cpu_baselines()
    if rank == 0:
        print(json.dumps(line), flush=True)
    replicas.finish(rk)
    return 0


def config0_rate(dev, steps: int = 1000) -> dict:
    """Config 0 (256 x 512, keep |k| <= 85, 1000 steps): device time of the
    plain single-run step with CUDA events (4-step graphs).  The state
    (100 MB for two buffers) fits in L2: a launch-and-latency figure, not a
    roofline one."""
    import torch

    from kh_simulations_b200.config import loads
    from kh_simulations_b200.run import KHRun

    run = KHRun(loads(CONFIG0), device=dev)
    run.init()
    stream = torch.cuda.Stream(device=dev)
    run.step(8, stream)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    run.step(steps, stream)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    cells = run.d.nx * run.d.nz
    run.close()
    return {"workload": "config 0: 256x512, keep |k| <= 85", "steps": steps, "ms_per_step": ms / steps,
            "value": cells * steps / (ms / 1e3), "unit": "cell-steps/s"}


def e2e_rate(run, args, stream, rk) -> dict:
    """Same metric through the public API with host buffers: upload the
    state from pinned host memory, K steps each followed by the energy
    read back (the reference's per-step diagnostic), download the state.
    Timed with CUDA events on the stream around all of it (host waits
    included), max over ranks."""
    import torch

    from kh_simulations_b200 import replicas

    st_host = run.state.to("cpu").pin_memory()
    out_host = torch.empty_like(st_host).pin_memory()
    torch.cuda.synchronize()
    replicas.barrier(rk)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    with torch.cuda.stream(stream):
        run.buf[0].copy_(st_host, non_blocking=True)
    run.lib.ymkh_set_current_buffer(run.ctx, 0)
    for _ in range(args.steps):
        run.step(1, stream)
        run.energy(stream)
    with torch.cuda.stream(stream):
        out_host.copy_(run.state, non_blocking=True)
    e1.record(stream)
    e1.synchronize()
    ms = replicas.max_over_ranks(e0.elapsed_time(e1), rk)
    cells = run.d.nx * run.d.nz
    sb = st_host.numel() * 8
    return {"value": replicas.aggregate_rate(cells * args.steps, ms, rk), "unit": "cell-steps/s",
            "h2d_bytes_per_step": sb / args.steps, "d2h_bytes_per_step": 8 + sb / args.steps,
            "note": "state uploaded once and downloaded once per K-step call; energy read back every step"}


SWEEP_BASE = "alpha_YM = 1.0\nrun_mode = 6\nlx_override = 20\n"


def _rel_l2_max(a, b) -> float:
    """Largest per-array relative L2 difference between two [24, NZ, NX] states."""
    d = (a - b).reshape(a.shape[0], -1).norm(dim=1)
    n = b.reshape(b.shape[0], -1).norm(dim=1).clamp_min(1e-300)
    return float((d / n).max())


def batch_by_size(dev) -> list:
    """Batched against plain for identical runs of one size at a time (filter
    off, CUDA events, one stream): where batching pays.  Sizes and counts:
    64 x 128x256, 64 x 256x512, 32 x 512x1024, 8 x 1024x2048."""
    import torch

    from kh_simulations_b200.batch import KHBatch
    from kh_simulations_b200.config import loads
    from kh_simulations_b200.run import KHRun
    from kh_simulations_b200.server import cfl_courant

    out = []
    for nz, nx, n, steps in [(128, 256, 64, 200), (256, 512, 64, 200), (512, 1024, 32, 100), (1024, 2048, 8, 40)]:
        ini = (SWEEP_BASE + "V0 = 0.05\neps_override = 1.0\nperturb_amp = 0.1\nk_mode = 1\n"
               f"nz_override = {nz}\nnx_override = {nx}\ncourant_override = {cfl_courant(nx, nz):.6f}\n")
        runs = [KHRun(loads(ini, f"size{i}"), device=dev) for i in range(n)]
        s = torch.cuda.Stream(device=dev)
        for r in runs:
            r.init(stream=s)
            r.step(4, s)
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        for r in runs:
            r.step(steps, s)
        e1.record(s)
        e1.synchronize()
        plain = e0.elapsed_time(e1)
        b = KHBatch(device=dev, graph_steps=4)
        for r in runs:
            b.add(r)
        b.step(4, s)
        torch.cuda.synchronize(dev)
        e0.record(s)
        b.step(steps, s)
        e1.record(s)
        e1.synchronize()
        bat = e0.elapsed_time(e1)
        cs = n * nz * nx * steps
        out.append({"runs": n, "grid": f"{nz}x{nx}", "steps": steps, "plain_cell_steps_per_s": cs / plain * 1e3,
                    "batched_cell_steps_per_s": cs / bat * 1e3, "batched_over_plain": plain / bat})
        b.close()
        for r in runs:
            r.close()
    return out


def batched_rate(args, dev, nruns: int, steps: int, check: int = 100) -> dict:
    """Config 2: the uneven sweep of `nruns` runs (seed 1; NZ 128..1024, NX
    256..2048) for `steps` steps each, with the energy checked every `check`
    steps and the reference's halt rule applied (NaN/Inf or E/E0 above the
    threshold, ymgpu2d/main_ym.cu:467-474): aggregate cell-steps/s of the
    batched form (one FCT and one Maxwell launch per step over every run's
    tiles, CUDA graphs; halted runs leave the batch) against the same runs
    stepped one after another through the plain single-run step, from the
    same state, timed with CUDA events on one stream around the whole pass
    (energy checks included).  Final states and halt steps of the two passes
    are compared run by run."""
    import math

    import torch

    from kh_simulations_b200.batch import KHBatch
    from kh_simulations_b200.run import KHRun
    from kh_simulations_b200.server import uneven_sweep

    stream = torch.cuda.Stream(device=dev)
    runs = [KHRun(c, device=dev) for c in uneven_sweep(1, nruns, SWEEP_BASE)]
    for r in runs:
        r.init(stream=stream)
        r.E0 = r.energy(stream)
        r.step(4, stream)  # warm-up: graphs captured, current buffer back to 0
    torch.cuda.synchronize(dev)
    s0 = [r.state.clone() for r in runs]

    def halted(r):
        e = r.energy(stream)
        return not math.isfinite(e) or e / r.E0 > r.d.energy_thresh

    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    plain_steps, plain_state = [], []
    cs_plain = 0
    e0.record(stream)
    for r in runs:
        done = 0
        while done < steps:
            k = min(check, steps - done)
            r.step(k, stream)
            done += k
            if halted(r):
                break
        plain_steps.append(done)
        cs_plain += done * r.d.nx * r.d.nz
    e1.record(stream)
    e1.synchronize()
    ms_plain = e0.elapsed_time(e1)
    plain_state = [r.state.clone() for r in runs]

    for r, s in zip(runs, s0):
        r.set_state(s)
    torch.cuda.synchronize(dev)
    batch = KHBatch(device=dev)
    for r in runs:
        batch.add(r)
    batch.step(4, stream)  # warm-up (graph capture); even, so every run is back on buffer 0
    torch.cuda.synchronize(dev)
    for r, s in zip(runs, s0):
        r.set_state(s)
    torch.cuda.synchronize(dev)
    live = list(runs)
    batch_steps = {id(r): 0 for r in runs}
    cs_batch = 0
    e0.record(stream)
    done = 0
    while done < steps and live:
        k = min(check, steps - done)
        batch.step(k, stream)
        done += k
        for r in list(live):
            batch_steps[id(r)] = done
            cs_batch += k * r.d.nx * r.d.nz
            if halted(r):
                batch.remove(r)
                live.remove(r)
    e1.record(stream)
    e1.synchronize()
    ms_batch = e0.elapsed_time(e1)
    dev_max = max(_rel_l2_max(r.state, p) for r, p in zip(runs, plain_state))
    same_halts = all(batch_steps[id(r)] == n for r, n in zip(runs, plain_steps))
    batch.close()
    cells = sum(r.d.nx * r.d.nz for r in runs)
    for r in runs:
        r.close()
    del runs, s0, plain_state
    torch.cuda.empty_cache()
    plain = cs_plain / (ms_plain / 1e3)
    batched = cs_batch / (ms_batch / 1e3)
    return {"workload": f"config 2: uneven sweep, {nruns} runs (seed 1), {cells} cells, {steps} steps, "
                        f"energy and halt rule every {check} steps",
            "batched_cell_steps_per_s": batched, "plain_cell_steps_per_s": plain, "batched_over_plain": batched / plain,
            "halted_runs": sum(n < steps for n in plain_steps), "same_halt_steps": same_halts,
            "max_rel_l2_batched_vs_plain": dev_max, "unit": "cell-steps/s",
            "timing": "CUDA events, one stream, around each whole pass"}


def _served_pass(dev, seconds, drain, step_scale, engine, large_cells):
    """One served and one sequential pass over the same seeded mix (seed 3):
    Poisson arrivals at 20 runs/s for `seconds` s, cells log-uniform in
    [128*256, 2048*4096], steps uniform in [2000, 20000] / step_scale, modes
    above NZ/3 subtracted with `engine`, 150 GB admission budget; each pass
    stops `drain` s after the last arrival at the latest."""
    from kh_simulations_b200.server import KHServer, poisson_mix

    def mix():
        return poisson_mix(3, 20.0, seconds, 128 * 256, 2048 * 4096, max(1, 2000 // step_scale),
                           max(2, 20000 // step_scale), SWEEP_BASE, keep_third=True, filter_engine=engine)

    import torch

    srv = KHServer(150 << 30, device=dev, chunk=50, large_cells=large_cells)
    gpu = dev.index if dev.index is not None else 0

    def one(fn):
        # each pass starts from an empty allocator cache, with its clocks sampled
        torch.cuda.synchronize(dev)
        torch.cuda.empty_cache()
        cs = ClockSampler(gpu)
        cs.start()
        rep = fn(mix(), deadline=seconds + drain)
        return rep, cs.stop()

    served, clk_a = one(srv.serve)
    seq, clk_b = one(srv.serve_sequential)
    a, b = served.summary(), seq.summary()
    a["clocks"], b["clocks"] = clk_a, clk_b
    keys = ("requests", "completed", "unfinished", "halted", "makespan_s", "cell_steps", "cell_steps_per_s",
            "p50_latency_s", "p99_latency_s", "clocks")
    # measured Amdahl bound: service time of the sequential pass split into
    # runs below / at or above large_cells; batching can at best remove the
    # former, since a large run fills the GPU alone
    t_small = sum(r.finished - r.admitted for r in seq.requests
                  if r.status in ("done", "halted") and r.cells < large_cells)
    t_large = sum(r.finished - r.admitted for r in seq.requests
                  if r.status in ("done", "halted") and r.cells >= large_cells)
    w = [(r.cells * r.steps, r.cells < large_cells) for r in mix()]
    return {"engine": engine, "served": {k: a[k] for k in keys}, "sequential": {k: b[k] for k in keys},
            "served_over_sequential": a["cell_steps_per_s"] / b["cell_steps_per_s"] if b["cell_steps_per_s"] else None,
            "p50_served_over_sequential": a["p50_latency_s"] / b["p50_latency_s"] if b["p50_latency_s"] else None,
            "small_runs_share_of_cell_steps": sum(x for x, sm in w if sm) / max(1, sum(x for x, _ in w)),
            "small_runs_share_of_sequential_time": t_small / max(1e-9, t_small + t_large),
            "amdahl_bound_served_over_sequential": (t_small + t_large) / t_large if t_large > 0 else None}


def _served_tolerance(dev, step_scale, nreq, large_cells):
    """Final states of the first `nreq` requests of the mix (seed 3, runs up
    to 1024 x 2048), served with the FP64 filter and with the TF32 filter,
    against the same requests run one by one plainly with the FP64 filter:
    the largest per-field relative L2 over requests and arrays, raw (over
    the field's own norm) and over the largest norm in the field's group."""
    import numpy as np

    from kh_simulations_b200.server import KHServer, poisson_mix

    groups = [range(0, 6), range(6, 9), range(9, 12), [12], [13, 14], range(15, 18), [18], [19, 20], range(21, 24)]

    def reqs(engine):
        out = [r for r in poisson_mix(3, 20.0, 30.0, 128 * 256, 2048 * 4096, max(1, 2000 // step_scale),
                                      max(2, 20000 // step_scale), SWEEP_BASE, keep_third=True,
                                      filter_engine=engine) if r.cells <= 1024 * 2048][:nreq]
        for r in out:
            r.arrival = 0.0
        return out

    srv = KHServer(150 << 30, device=dev, chunk=50, keep_state=True, large_cells=large_cells)
    plain = reqs("dft")
    srv.serve_sequential(plain)
    res = {}
    for engine in ("dft", "tf32x3"):
        rs = reqs(engine)
        srv.serve(rs)
        raw = grp = 0.0
        for a, b in zip(rs, plain):
            if a.status != "done" or b.status != "done":
                continue
            num = np.sqrt(((a.state - b.state) ** 2).reshape(24, -1).sum(1))
            nrm = np.sqrt((b.state ** 2).reshape(24, -1).sum(1))
            raw = max(raw, float(np.max(np.where(nrm > 0, num / np.where(nrm > 0, nrm, 1), num))))
            for g in groups:
                g = list(g)
                grp = max(grp, float(num[g].max() / max(nrm[g].max(), 1e-300)))
        res[engine] = {"max_rel_l2_vs_fp64_plain_raw": raw, "max_rel_l2_vs_fp64_plain_group": grp,
                       "within_1e-10": raw <= 1e-10,
                       "requests": [f"{derive_grid(r)} x {r.steps} steps ({r.status})" for r in rs]}
    return res


def derive_grid(req) -> str:
    from kh_simulations_b200.config import derive

    d = derive(req.cfg)
    return f"{d.nz}x{d.nx}"


def served_rate(args, dev, seconds: float) -> dict:
    """Served request mix with config 4's distributions (Poisson 20 runs/s,
    cells log-uniform in [128*256, 2048*4096], kz = 0 suppressed in every
    other request, modes above NZ/3 subtracted) over a `seconds`-long arrival
    window, steps scaled down by --served-step-scale, each pass bounded to
    --served-drain s after the last arrival (unfinished runs count their
    steps and their latency is censored there).  The full mix offers about
    200 times what one B200 steps per second; the scaled one still offers
    more than its capacity, so both passes run saturated and their
    throughputs compare capacities.  Continuous batching (KHServer.serve:
    runs of 2^20 cells and more stepped alone in arrival order on their own
    stream, the smaller ones batched beside them) against the same requests
    one by one through the plain step (serve_sequential).  The TF32 filter
    (config 4's split precision) is the headline; the FP64 filter pass keeps
    the 1e-10 bar; a tolerance leg compares final states of both served
    forms with the plain FP64 runs."""
    large = 1 << 20
    out = {"workload": f"Poisson 20/s for {seconds:g} s (seed 3), 128x256..2048x4096 cells, "
                       f"{2000 // args.served_step_scale}..{20000 // args.served_step_scale} steps "
                       f"(config 4's 2000..20000 / {args.served_step_scale}), 150 GB budget, keep |k| <= NZ/3, "
                       f"passes bounded at {args.served_drain:g} s after the last arrival",
           "large_cells": large, "unit": "cell-steps/s",
           "latency_clock": "host wall clock (arrival to completion; unfinished runs censored at the bound)"}
    out["tf32x3"] = _served_pass(dev, seconds, args.served_drain, args.served_step_scale, "tf32x3", large)
    if args.served_fp64_seconds > 0:
        out["dft"] = _served_pass(dev, args.served_fp64_seconds, args.served_drain, args.served_step_scale, "dft",
                                  large)
    if args.served_check > 0:
        tol = _served_tolerance(dev, args.served_step_scale, args.served_check, large)
        out["tolerance"] = tol
        out["tf32x3"]["max_rel_l2_vs_fp64_plain"] = tol["tf32x3"]["max_rel_l2_vs_fp64_plain_raw"]
        out["tf32x3"]["within_metric_1e-10"] = tol["tf32x3"]["within_1e-10"]
        if "dft" in out:
            out["dft"]["max_rel_l2_vs_fp64_plain"] = tol["dft"]["max_rel_l2_vs_fp64_plain_raw"]
            out["dft"]["within_metric_1e-10"] = tol["dft"]["within_1e-10"]
    return out


def measured_tf32_peak() -> tuple:
    """TF32 dense tensor rate: half the measured bf16 dense burst rate (the
    B200's TF32 rate is half its bf16 rate); without MEASURED_PEAKS.json,
    half of the profiling recipe's fallback bf16 figure (1.59 PFLOP/s)."""
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        if "bf16_tflops" in d:
            return float(d["bf16_tflops"]) / 2.0, "half of measured bf16 dense"
    return 1590.0 / 2.0, "half of fallback bf16 dense (1.59 PFLOP/s)"


def filter_engines(args, dev) -> dict:
    """The DFT band filter at the split-precision configuration's size (one
    run at NZ 1024 x NX 2048, keep |k| <= NZ/3: modes 342..512 subtracted, 21
    arrays): band-stage device time with the FP64 filter and with the 3-pass
    TF32 tensor-core filter, the step time with each, and the tensor
    roofline of the TF32 filter."""
    import torch

    from kh_simulations_b200 import _lib
    from kh_simulations_b200.config import loads
    from kh_simulations_b200.run import KHRun

    wl = "kh_1024x2048"
    out = {"workload": f"{wl}, keep |k| <= NZ/3, 21 filtered arrays", "bands_ms": {}, "step_ms": {}}
    lib = _lib.load()
    bands = None
    for eng in ("dft", "tf32x3"):
        run = KHRun(loads(ini_for(wl, "keep", eng)), device=dev)
        run.init()
        stream = torch.cuda.Stream(device=dev)
        t = (C.c_float * 8)()
        _lib.check(lib.ymkh_stage_times(run.ctx, 3, C.c_void_p(stream.cuda_stream), t, 8), "stage times")
        n = 10
        _lib.check(lib.ymkh_stage_times(run.ctx, n, C.c_void_p(stream.cuda_stream), t, 8), "stage times")
        out["bands_ms"][eng] = t[4] / n
        out["step_ms"][eng] = sum(t[:7]) / n
        bands = run.d.bands
        nx, nz = run.d.nx, run.d.nz
        run.close()
    # algorithmic flops of the two contractions per band and array
    flops = sum(2 * 2.0 * (2 * (hi - lo + 1)) * nx * nz * 21 for lo, hi in bands)
    peak, kind = measured_tf32_peak()
    ms = out["bands_ms"]["tf32x3"]
    achieved = flops / (ms / 1e3) / 1e12
    out["speedup_tf32x3_over_dft"] = out["bands_ms"]["dft"] / ms
    out["roofline_tf32x3"] = {"bound": "tensor", "achieved": achieved, "executed": 3 * achieved, "peak": peak,
                              "unit": "TFLOP/s", "frac": 3 * achieved / peak, "peak_source": kind,
                              "note": "achieved = algorithmic flops / band-stage time; executed counts the 3 passes"}
    return out


def filter_error(args, dev, steps: int, nruns: int, control: bool = False) -> dict:
    """Error of the 3-pass TF32 filter against the FP64 filter, from the same
    initial state, on `nruns` runs at NZ 1024 x NX 2048 (seed 2,
    uneven-sweep parameter ranges, keep |k| <= NZ/3).  Both engines step in
    lockstep in chunks of 100 until `steps` or until either meets the
    reference's halt rule (NaN/Inf or E/E0 above the threshold,
    ymgpu2d/main_ym.cu:467-474); the per-field relative L2 of the state and
    the relative error of the k_mode amplitude are taken at the last chunk
    both completed.  With `control`, both runs use the FP64 filter and the
    second starts with the beam-A density (about 1 everywhere) scaled by
    1 + 2^-52, one ulp: how far two FP64 trajectories part from a
    rounding-level difference."""
    import math

    import numpy as np
    import torch

    from kh_simulations_b200._lib import STATE_NAMES
    from kh_simulations_b200.run import KHRun
    from kh_simulations_b200.server import split_precision_runs

    # groups of arrays sharing a scale (E, By, Az, n, p, Q of each beam): an
    # array's error is divided by its group's largest norm, as in the parity
    # tests (some arrays are pure cancellation residues beside their group)
    groups = [range(0, 6), range(6, 9), range(9, 12), [12], [13, 14], range(15, 18), [18], [19, 20], range(21, 24)]
    checkpoints = sorted({c for c in (1, 100, 1000, 2000, steps) if c <= steps})
    table = {c: np.zeros(24) for c in checkpoints}
    amp = {c: 0.0 for c in checkpoints}
    reached = []
    for cfg in split_precision_runs(2, nruns, SWEEP_BASE):
        runs = {}
        for eng in ("dft", "tf32x3"):
            cfg.filter_engine = "dft" if control else eng
            r = KHRun(cfg, device=dev)
            r.init()
            if control and eng == "tf32x3":
                r.state[STATE_NAMES.index("nA")] *= 1.0 + 2.0 ** -52
            r.E0 = r.energy()
            runs[eng] = r
        done = 0
        for c in checkpoints:
            k = c - done
            ok = True
            while k > 0 and ok:
                kk = min(100, k)
                for r in runs.values():
                    r.step(kk)
                    e = r.energy()
                    ok = ok and math.isfinite(e) and e / r.E0 <= r.d.energy_thresh
                k -= kk
            if not ok:
                break
            done = c
            a, b = runs["tf32x3"].state, runs["dft"].state
            d = (a - b).reshape(24, -1).norm(dim=1).cpu().numpy()
            n = b.reshape(24, -1).norm(dim=1).cpu().numpy()
            for g in groups:
                g = list(g)
                scale = max(n[g].max(), 1e-300)
                table[c][g] = np.maximum(table[c][g], d[g] / scale)
            ma, mb = runs["tf32x3"].mode_amp()[0], runs["dft"].mode_amp()[0]
            amp[c] = max(amp[c], abs(ma - mb) / max(abs(mb), 1e-300))
        reached.append(done)
        for r in runs.values():
            r.close()
        torch.cuda.empty_cache()
    return {"workload": f"{nruns} runs at 1024x2048 (seed 2), keep |k| <= NZ/3, up to {steps} steps"
                        + (", control: FP64 against FP64 with nA scaled by 1+2^-52" if control else ""),
            "steps_reached": reached, "metric": "per-array rel-L2, divided by the largest norm in its group",
            "max_rel_l2_by_step": {str(c): {STATE_NAMES[i]: float(table[c][i]) for i in range(24)} for c in checkpoints},
            "max_rel_mode_amp_err_by_step": {str(c): amp[c] for c in checkpoints},
            "reference": "the FP64 filter (matches the oracle to 1e-12 per step)"}


def filter_keep_rate(args, dev) -> dict:
    """The workload as config 1 states it, filter on: modes above NZ/3
    subtracted every step (at NZ = 4096, modes 1366..2048 of 21 arrays), with
    the FP64 DFT engine and with the 3-pass TF32 tensor-core engine.  For
    each: step time (CUDA events over plain steps), cell-steps/s and the band
    stage's share; for TF32, the band stage's tensor roofline (algorithmic
    flops of the two contractions per array over its device time, and 3x that
    executed, against half the measured bf16 dense rate) and its error
    against the FP64 engine after one step from the same state (per-field
    relative L2, raw and over the largest norm in the field's group)."""
    import numpy as np
    import torch

    from kh_simulations_b200 import _lib
    from kh_simulations_b200.config import loads
    from kh_simulations_b200.run import KHRun

    lib = _lib.load()
    out = {"workload": f"{args.workload}, keep |k| <= NZ/3 (config 1 as stated), 21 filtered arrays"}
    states = {}
    groups = [range(0, 6), range(6, 9), range(9, 12), [12], [13, 14], range(15, 18), [18], [19, 20], range(21, 24)]
    s0 = None
    for eng, nsteps in (("dft", 2), ("tf32x3", 4)):
        run = KHRun(loads(ini_for(args.workload, "keep", eng)), device=dev)
        run.init()
        stream = torch.cuda.Stream(device=dev)
        if s0 is None:
            s0 = run.state.clone()
        t = (C.c_float * 8)()
        _lib.check(lib.ymkh_stage_times(run.ctx, 1, C.c_void_p(stream.cuda_stream), t, 8), "stage times")
        _lib.check(lib.ymkh_stage_times(run.ctx, nsteps, C.c_void_p(stream.cuda_stream), t, 8), "stage times")
        step_ms = sum(t[:7]) / nsteps
        bands_ms = t[4] / nsteps
        cells = run.d.nx * run.d.nz
        bands = run.d.bands
        flops = sum(2 * 2.0 * (2 * (hi - lo + 1)) * run.d.nx * run.d.nz * 21 for lo, hi in bands)
        r = {"ms_per_step": step_ms, "cell_steps_per_s": cells / (step_ms / 1e3), "bands_ms": bands_ms,
             "band_share": bands_ms / step_ms, "bands": bands,
             "band_algorithmic_tflops": flops / (bands_ms / 1e3) / 1e12}
        if eng == "tf32x3":
            peak, kind = measured_tf32_peak()
            ach = r["band_algorithmic_tflops"]
            r["roofline"] = {"bound": "tensor", "achieved": ach, "executed": 3 * ach, "peak": peak,
                             "unit": "TFLOP/s", "frac": 3 * ach / peak, "peak_source": kind}
        # one step from the common initial state, for the error of TF32 against FP64
        run.set_state(s0)
        run.step(1, stream)
        torch.cuda.synchronize(dev)
        states[eng] = run.state.clone()
        out[eng] = r
        run.close()
        del run
        torch.cuda.empty_cache()
    a, b = states["tf32x3"], states["dft"]
    num = (a - b).reshape(24, -1).norm(dim=1).cpu().numpy()
    nrm = b.reshape(24, -1).norm(dim=1).cpu().numpy()
    raw = np.where(nrm > 0, num / np.where(nrm > 0, nrm, 1), num)
    grp = np.zeros(24)
    for g in groups:
        g = list(g)
        grp[g] = num[g] / max(nrm[g].max(), 1e-300)
    out["tf32x3"]["error_vs_dft_after_1_step"] = {"max_raw": float(raw.max()), "max_group": float(grp.max()),
                                                  "median_raw": float(np.median(raw))}
    out["tf32x3_over_dft"] = out["dft"]["ms_per_step"] / out["tf32x3"]["ms_per_step"]
    del states, s0, a, b
    torch.cuda.empty_cache()
    return out


if __name__ == "__main__":
    sys.exit(main())
