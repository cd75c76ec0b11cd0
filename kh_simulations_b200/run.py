"""``KHRun``: one Kelvin–Helmholtz run with its state resident in HBM.

Replaces the driver ymgpu2d/main_ym.cu: configuration and derivation
(:24-83), allocation (:85-121, here two 24-array FP64 buffers held as torch
tensors), seed profile upload (:178-217), initial state (:219-237), the
step loop with the energy check and halt rules (:318-479), ``energy.csv``
in the reference's format (:251-256, :458-466) and the state snapshots
(:260-313, :476-477).
The arithmetic runs in the CUDA library (include/ymkh.h); this module only
owns memory, streams and files.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass
from pathlib import Path

import numpy as np
import torch

from . import _lib
from ._lib import GAUSS_NOUT, NSTATE, PAIRS, SNAP_CSV, SNAP_FP64, STATE_NAMES, Grid, InitParams, check
from .config import Derived, RunConfig, derive, load_config, step_params
from .seed import interpolate, load_profiles


def init_params(cfg: RunConfig, d: Derived, profiles: dict | None = None):
    """ymkh_init_params for the run (arguments of kernel_ym_init at
    ymgpu2d/main_ym.cu:223-225).  Returns (params, arrays to keep alive)."""
    ip = InitParams()
    ip.run_mode, ip.k_mode = cfg.run_mode, cfg.k_mode
    ip.perturb_amp, ip.V0, ip.epsilon = cfg.perturb_amp, d.V0, d.eps
    ip.alpha_YM, ip.init_by1_eq, ip.vz_edge_taper = d.alpha, cfg.init_by1_eq, cfg.vz_edge_taper
    keep = []
    for k, v in (profiles or {}).items():
        arr = np.ascontiguousarray(v, dtype=np.float64)
        if arr.shape != (d.nx,):
            raise ValueError(f"seed profile {k} has shape {arr.shape}, expected ({d.nx},)")
        keep.append(arr)
        setattr(ip, "seed_" + k, arr.ctypes.data)
    return ip, keep


def _stream_ptr(stream) -> int | None:
    if stream is None:
        return torch.cuda.current_stream().cuda_stream
    return stream.cuda_stream


@dataclass
class EnergyRecord:
    step: int
    time: float
    energy: float
    ratio: float
    mode_amp: float = math.nan  # k_mode amplitude of Az2 + i Az3 (when recorded)


CHECKPOINT_VERSION = 1


class KHRun:
    """One run.  ``state`` is a [24, NZ, NX] float64 CUDA tensor (include/ymkh.h order)."""

    def __init__(self, cfg: RunConfig, device: int | str | torch.device = "cuda", *, graph_steps: int | None = None,
                 fct_shape: tuple | None = None, tune: bool = False):
        if not torch.cuda.is_available():
            raise _lib.YMKHError("KHRun needs a CUDA device (no CPU fallback)")
        self.cfg = cfg
        self.d: Derived = derive(cfg)
        self.device = torch.device(device)
        self.lib = _lib.load()
        nx, nz = self.d.nx, self.d.nz
        with torch.cuda.device(self.device):
            self.buf = [torch.zeros((NSTATE, nz, nx), dtype=torch.float64, device=self.device) for _ in range(2)]
            grid = Grid(nx, nz, self.d.dx, self.d.dz)
            self.params = step_params(cfg, self.d)
            ctx = C.c_void_p()
            check(self.lib.ymkh_create(C.byref(grid), C.byref(self.params), C.byref(ctx)), "ymkh_create")
            self.ctx = ctx
            p0 = (C.c_void_p * NSTATE)(*[self.buf[0][i].data_ptr() for i in range(NSTATE)])
            p1 = (C.c_void_p * NSTATE)(*[self.buf[1][i].data_ptr() for i in range(NSTATE)])
            check(self.lib.ymkh_bind_state2(self.ctx, p0, p1), "ymkh_bind_state2")
            if graph_steps is not None:
                check(self.lib.ymkh_set_graph_steps(self.ctx, graph_steps), "ymkh_set_graph_steps")
            if fct_shape is not None:
                check(self.lib.ymkh_set_fct_shape(self.ctx, *fct_shape), "ymkh_set_fct_shape")
            elif tune:
                from . import autotune

                autotune.apply(self)
        self.step_count = 0
        self.E0: float | None = None
        self.history: list[EnergyRecord] = []
        self.halted = False
        self.halt_reason = ""

    # ---------------------------------------------------------------- state
    @property
    def current(self) -> int:
        return int(self.lib.ymkh_current_buffer(self.ctx))

    @property
    def state(self) -> torch.Tensor:
        """The current state buffer (a view; valid until the next step)."""
        return self.buf[self.current]

    def fct_shape(self) -> tuple:
        """(FCT strip width in threads per beam, z-segment rows) in use."""
        tx, seg = C.c_int(), C.c_int()
        check(self.lib.ymkh_get_fct_shape(self.ctx, C.byref(tx), C.byref(seg)), "ymkh_get_fct_shape")
        return tx.value, seg.value

    def field(self, name: str) -> torch.Tensor:
        return self.state[STATE_NAMES.index(name)]

    def set_state(self, st) -> None:
        """Copy a [24, NZ, NX] array (numpy or torch) into the current buffer."""
        t = torch.as_tensor(st, dtype=torch.float64)
        if tuple(t.shape) != (NSTATE, self.d.nz, self.d.nx):
            raise ValueError(f"state shape {tuple(t.shape)} != {(NSTATE, self.d.nz, self.d.nx)}")
        check(self.lib.ymkh_set_current_buffer(self.ctx, 0), "ymkh_set_current_buffer")
        self.buf[0].copy_(t.to(self.device))

    def state_numpy(self) -> np.ndarray:
        torch.cuda.synchronize(self.device)
        return self.state.cpu().numpy()

    # ----------------------------------------------------------------- init
    def init(self, seed_file: str | Path | None = None, stream=None, seed_profiles: dict | None = None) -> None:
        """kernel_ym_init with the run's parameters (main_ym.cu:219-226).

        The seed profiles come from, in this order: ``seed_profiles`` (float32
        profiles on any grid, as a seed file holds them), ``seed_file``,
        the config's ``seed_profile_file``, or, with ``eigen_seed = 1``, the
        eigenmode of the run's parameters solved here (eigenmode.py) as the
        reference's offline solver would write it.  Profiles are interpolated
        to the run's grid as the reference interpolates a seed file."""
        cfg, d = self.cfg, self.d
        seed_file = seed_file if seed_file is not None else (cfg.seed_profile_file or None)
        if seed_profiles is None and seed_file is None and cfg.eigen_seed:
            from . import eigenmode

            seed_profiles = eigenmode.cached_seed(eigenmode.spec_for_run(cfg, d, cfg.eigen_seed_nx))
        if seed_profiles is not None:
            profiles = {k: interpolate(v, d.nx) for k, v in seed_profiles.items()}
        else:
            profiles = load_profiles(seed_file, d.nx) if seed_file else None
        ip, keep = init_params(cfg, d, profiles)
        with torch.cuda.device(self.device):
            cur = torch.cuda.current_stream(self.device)
            if stream is not None:  # after the buffers' zero fill on torch's current stream
                stream.wait_stream(cur)
            check(self.lib.ymkh_init(self.ctx, C.byref(ip), C.c_void_p(_stream_ptr(stream))), "ymkh_init")
            # the state is ready on return; other streams' work is not waited for
            (stream if stream is not None else cur).synchronize()
        self.step_count = 0
        self.history.clear()
        self.halted = False
        self.E0 = None

    def add_noise(self, sigma: float = 1e-6, seed: int = 0, names=("Ex1", "Ex2", "Ex3", "Ez1", "Ez2", "Ez3",
                                                                   "By1", "By2", "By3")) -> None:
        """Optional N(0, sigma) field noise, drawn on the host from numpy's
        default_rng(seed) in the given array order, then uploaded (so that a
        CPU check sees the same numbers)."""
        rng = np.random.default_rng(seed)
        st = self.state
        for nm in names:
            noise = rng.normal(0.0, sigma, size=(self.d.nz, self.d.nx))
            st[STATE_NAMES.index(nm)] += torch.from_numpy(noise).to(self.device)

    # ----------------------------------------------------------------- step
    def step(self, n: int = 1, stream=None) -> None:
        with torch.cuda.device(self.device):
            check(self.lib.ymkh_step(self.ctx, int(n), C.c_void_p(_stream_ptr(stream))), "ymkh_step")
        self.step_count += n

    def energy(self, stream=None) -> float:
        out = C.c_double()
        with torch.cuda.device(self.device):
            check(self.lib.ymkh_energy(self.ctx, C.byref(out), C.c_void_p(_stream_ptr(stream))), "ymkh_energy")
        return out.value

    def mode_amp(self, k: int | None = None, stream=None) -> tuple:
        out = (C.c_double * 2)()
        k = self.cfg.k_mode if k is None else k
        with torch.cuda.device(self.device):
            check(self.lib.ymkh_mode_amp(self.ctx, int(k), out, C.c_void_p(_stream_ptr(stream))), "ymkh_mode_amp")
        return out[0], out[1]

    def circ_amp(self, pair: str = "Az", k: int | None = None, weight=None, stream=None) -> tuple:
        """(|F2 + i F3|_k, |F2 - i F3|_k) averaged over x for F in Az, By, Ex,
        Ez: the plain mean, or the sum weighted by ``weight`` (NX values,
        e.g. growth.xi_weight, as in ymgpu2d/analysis/resolution_convergence.py:77-86)."""
        out = (C.c_double * 2)()
        k = self.cfg.k_mode if k is None else k
        w = None
        if weight is not None:
            w = np.ascontiguousarray(weight, dtype=np.float64)
            if w.shape != (self.d.nx,):
                raise ValueError(f"weight has shape {w.shape}, expected ({self.d.nx},)")
        with torch.cuda.device(self.device):
            check(self.lib.ymkh_circ_amp(self.ctx, PAIRS[pair], int(k), None if w is None else w.ctypes.data, out,
                                         C.c_void_p(_stream_ptr(stream))), "ymkh_circ_amp")
        return out[0], out[1]

    def gauss(self, stream=None) -> dict:
        """Root-mean-square terms of the non-Abelian Gauss law on the current
        state (ymgpu2d/analysis/gauss_check.py:40-110 and its summary):
        arrays of the three colours for G, div_E, nonabelian, rho and lhs
        (div_E + nonabelian), and Etot_scale = rms(|Ex|+|Ez| summed over
        colours) / dx + 1e-30, the scale of its relative error."""
        out = (C.c_double * GAUSS_NOUT)()
        with torch.cuda.device(self.device):
            check(self.lib.ymkh_gauss(self.ctx, out, C.c_void_p(_stream_ptr(stream))), "ymkh_gauss")
        v = np.array(out[:], dtype=np.float64)
        return {"G": v[0:3], "div_E": v[3:6], "nonabelian": v[6:9], "rho": v[9:12], "lhs": v[12:15],
                "Etot_scale": v[15] / self.d.dx + 1e-30}

    def snapshot(self, path: str | Path, fmt: str = "csv", stream=None) -> None:
        """Write the current state to ``path`` in the background: ``csv`` is
        the reference's 26-column snapshot, ``fp64`` the exact binary form
        (include/ymkh.h, ymkh_snapshot).  snapshot_wait() joins the writers."""
        f = {"csv": SNAP_CSV, "fp64": SNAP_FP64}[fmt]
        with torch.cuda.device(self.device):
            check(self.lib.ymkh_snapshot(self.ctx, str(path).encode(), f, C.c_void_p(_stream_ptr(stream))),
                  "ymkh_snapshot")

    def snapshot_wait(self) -> None:
        check(self.lib.ymkh_snapshot_wait(self.ctx), "ymkh_snapshot_wait")

    # ------------------------------------------------------------------ loop
    def run(self, total_steps: int | None = None, energy_stride: int | None = None, csv: str | Path | None = None,
            on_energy=None, stream=None, mode_amp: bool = False, export_dir: str | Path | None = None,
            export_format: str = "csv", export_stride: int | None = None, on_export=None) -> list:
        """The time loop of ymgpu2d/main_ym.cu:318-479: energy every
        ``energy_stride`` steps, halt on NaN/Inf or E/E0 above the
        reference's threshold (:249, :467-474).  With mode_amp, the k_mode
        amplitude (offline in the reference,
        analysis/remote_timeseries.py:62-77) is recorded at the same stride.
        Every ``export_stride`` steps (and at step 0), after the energy
        check, the state is exported (:476-477): written to
        ``export_dir/ym_%06d.csv`` (or ``.fp64``) when export_dir is given,
        and passed to ``on_export(run, step)`` when that is given."""
        loop = RunLoop(self, total_steps, energy_stride, csv, on_energy, stream, mode_amp, export_dir, export_format,
                       export_stride, on_export)
        try:
            loop.start()
            while not loop.finished:
                self.step(loop.steps_to_event(), stream)
                loop.after_steps()
        finally:
            loop.close()
        return self.history

    # ------------------------------------------------------------ checkpoint
    def save_checkpoint(self, path: str | Path) -> None:
        """Raw FP64 state and loop position (.npz): the 24 arrays in
        include/ymkh.h order, the step count, E0, the halt flag and the
        energy history.  The reference has no checkpoint (its snapshots are
        6-digit CSV, ymgpu2d/main_ym.cu:290-306); this one is exact, so a run
        resumed from it continues bit for bit."""
        h = self.history
        np.savez(Path(path), version=CHECKPOINT_VERSION, state=self.state_numpy(), nx=self.d.nx, nz=self.d.nz,
                 step_count=self.step_count, E0=np.nan if self.E0 is None else self.E0,
                 halted=self.halted, halt_reason=self.halt_reason,
                 hist=np.array([[r.step, r.time, r.energy, r.ratio, r.mode_amp] for r in h], dtype=np.float64)
                 .reshape(len(h), 5))

    def load_checkpoint(self, path: str | Path) -> None:
        """Restore a checkpoint written by save_checkpoint for the same grid."""
        with np.load(Path(path), allow_pickle=False) as z:
            if int(z["version"]) != CHECKPOINT_VERSION:
                raise ValueError(f"checkpoint version {int(z['version'])} != {CHECKPOINT_VERSION}")
            if (int(z["nx"]), int(z["nz"])) != (self.d.nx, self.d.nz):
                raise ValueError(f"checkpoint grid {int(z['nz'])}x{int(z['nx'])} != {self.d.nz}x{self.d.nx}")
            self.set_state(z["state"])
            self.step_count = int(z["step_count"])
            e0 = float(z["E0"])
            self.E0 = None if math.isnan(e0) else e0
            self.halted = bool(z["halted"])
            self.halt_reason = str(z["halt_reason"])
            self.history = [EnergyRecord(int(r[0]), float(r[1]), float(r[2]), float(r[3]), float(r[4]))
                            for r in z["hist"]]
        torch.cuda.synchronize(self.device)

    def close(self) -> None:
        """Free the context and drop the state buffers (back to torch's cache)."""
        if getattr(self, "ctx", None):
            self.lib.ymkh_destroy(self.ctx)
            self.ctx = None
        self.buf = []

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass

    @classmethod
    def from_ini(cls, path: str | Path, **kw) -> "KHRun":
        return cls(load_config(path), **kw)


class RunLoop:
    """The bookkeeping of ymgpu2d/main_ym.cu:318-479 for one run, with the
    stepping left to the caller (``KHRun.run`` steps the run alone; a
    campaign steps many runs in one batch).  ``steps_to_event`` says how
    many steps may be taken before the next energy check, export or the
    end; ``after_steps`` does what the reference does at the step reached:
    energy check, energy.csv line, halt rule, then export."""

    def __init__(self, run: KHRun, total_steps=None, energy_stride=None, csv=None, on_energy=None, stream=None,
                 mode_amp=False, export_dir=None, export_format="csv", export_stride=None, on_export=None):
        d = run.d
        self.run = run
        self.total = d.total_steps if total_steps is None else total_steps
        self.stride = d.energy_stride if energy_stride is None else energy_stride
        self.xstride = d.export_stride if export_stride is None else export_stride
        self.stream = stream
        self.mode_amp = mode_amp
        self.on_energy = on_energy
        self.on_export = on_export
        self.export_dir = Path(export_dir) if export_dir is not None else None
        self.export_format = export_format
        self.exporting = export_dir is not None or on_export is not None
        if self.export_dir is not None:
            self.export_dir.mkdir(parents=True, exist_ok=True)
        self.fh = open(csv, "w") if csv else None

    @property
    def finished(self) -> bool:
        return self.run.step_count >= self.total or self.run.halted

    def _export(self, step: int) -> None:
        if self.export_dir is not None:
            self.run.snapshot(self.export_dir / f"ym_{step:06d}.{self.export_format}", self.export_format, self.stream)
        if self.on_export:
            self.on_export(self.run, step)

    def start(self) -> None:
        run, fh = self.run, self.fh
        if run.E0 is None:
            run.E0 = run.energy(self.stream)
            amp0 = run.mode_amp(stream=self.stream)[0] if self.mode_amp else math.nan
            run.history.append(EnergyRecord(0, 0.0, run.E0, 1.0, amp0))
            if fh:
                fh.write("step,time,E_total,E_ratio\n")
                fh.write(f"0,0,{run.E0:.8e},1.0\n")
            if self.exporting and run.step_count == 0:
                self._export(0)

    def steps_to_event(self) -> int:
        sc = self.run.step_count
        n = min(self.stride - sc % self.stride, self.total - sc)
        if self.exporting:
            n = min(n, self.xstride - sc % self.xstride)
        return n

    def after_steps(self) -> None:
        run, d, sc = self.run, self.run.d, self.run.step_count
        if sc % self.stride == 0:
            E = run.energy(self.stream)
            ratio = E / run.E0
            t = sc * d.dt
            amp = run.mode_amp(stream=self.stream)[0] if self.mode_amp else math.nan
            rec = EnergyRecord(sc, t, E, ratio, amp)
            run.history.append(rec)
            if self.fh:
                self.fh.write(f"{sc},{t:.8e},{E:.8e},{ratio:.8e}\n")
                self.fh.flush()
            if self.on_energy:
                self.on_energy(run, rec)
            if math.isnan(E) or math.isinf(E):
                run.halted, run.halt_reason = True, f"NaN/Inf at t={t}"
            elif ratio > d.energy_thresh:
                run.halted, run.halt_reason = True, f"E/E0={ratio} > {d.energy_thresh} at t={t}"
        if self.exporting and sc % self.xstride == 0:
            self._export(sc)

    def close(self) -> None:
        if self.fh:
            self.fh.close()
            self.fh = None
        if self.export_dir is not None:
            self.run.snapshot_wait()
