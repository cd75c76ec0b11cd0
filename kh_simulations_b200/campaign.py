"""Campaigns: many configurations run as one batched job on one GPU.

The reference runs a campaign as a shell script (ymgpu2d/scripts/*.sh,
written by ymgpu2d/analysis/gen_*_campaign.py).  For each configuration the
script writes an .ini through a heredoc and runs ``ym_coupled`` on it, one
process after another.  Two offline steps follow:
ymgpu2d/analysis/remote_timeseries.py reads each run's CSV snapshots into
the k_mode amplitude series ``timeseries_k<kz>.csv``, and
ymgpu2d/analysis/batch_analyze.py fits growth rates into
``batch_results.csv``.

Here ``parse_campaign_script`` reads the .ini texts of such a script in run
order, and ``CampaignRunner`` runs them all in one process through one
``KHBatch`` with FIFO admission by device footprint:
- every run keeps the reference's loop exactly (``run.RunLoop``): energy
  check and halt rule at its own energy stride, ``energy.csv``, exports at
  its own export stride (ymgpu2d/main_ym.cu:244-249, 457-477), in the
  output directory the reference would name (main_ym.cu:143-176);
- at each export the amplitude |Az2 + i Az3| at k_mode is measured on the
  device, with no snapshot written, and ``timeseries_k<kz>.csv`` is written
  as remote_timeseries.py writes it;
- when the run ends, its growth rate is fitted as batch_analyze.py fits it,
  and one row per run goes to ``batch_results.csv``.

The batch steps all resident runs together up to the nearest event of any
of them (an energy check, an export or an end).  A batched step is
bit-identical to the run's own step, so every file a run writes here is
the file that ``KHRun.run`` alone would write.
"""
from __future__ import annotations

import argparse
import csv
import math
import re
import shlex
import time
from collections import deque
from dataclasses import dataclass, field
from pathlib import Path

from . import growth
from .config import RunConfig, derive, loads, out_dir_name
from .server import footprint


@dataclass
class CampaignRun:
    name: str   # the .ini path the script writes, without directory or suffix
    ini: str    # the .ini text
    order: int  # position in the script's run sequence


_HEREDOC = re.compile(r"""cat\s*>\s*(\S+)\s*<<-?\s*(['"]?)(\w+)\2""")


def parse_campaign_script(text: str) -> list:
    """The runs of a campaign shell script, in the order it runs them.

    A run is an ``.ini`` written by a heredoc (``cat > PATH <<'TAG'`` ...
    ``TAG``) and later passed to ``ym_coupled``.  An .ini path written more
    than once runs with the text written last before its ``ym_coupled``
    line; .ini files that are never run are ignored."""
    inis: dict = {}
    runs = []
    lines = text.splitlines()
    i = 0
    while i < len(lines):
        line = lines[i]
        m = _HEREDOC.search(line)
        if m:
            path, tag = m.group(1), m.group(3)
            body = []
            i += 1
            while i < len(lines) and lines[i].strip() != tag:
                body.append(lines[i].strip())
                i += 1
            inis[path] = "\n".join(body) + "\n"
            i += 1
            continue
        if "ym_coupled" in line:
            try:
                words = shlex.split(line, comments=True)
            except ValueError:
                words = line.split()
            for j, w in enumerate(words):
                if w.endswith("ym_coupled") and j + 1 < len(words) and words[j + 1] in inis:
                    p = words[j + 1]
                    runs.append(CampaignRun(Path(p).stem, inis[p], len(runs)))
        i += 1
    return runs


def kz_label(kz: float) -> str:
    """Wavenumber label of the timeseries file name: 1 -> '1', 1.5 -> '1p5',
    0.125 -> '0p125' (ymgpu2d/analysis/batch_analyze.py:181-186)."""
    kz = round(kz, 3)
    if kz == int(kz):
        return str(int(kz))
    return f"{kz:.3f}".rstrip("0").replace(".", "p")


RESULT_COLUMNS = ("kz", "alpha", "V0", "xi_sponge", "gamma_sim", "gamma_exact", "ratio", "R2", "t0", "t1",
                  "has_plateau", "gamma_plateau", "plateau_t0", "plateau_t1", "plateau_ratio", "source", "node")


def result_row(cfg: RunConfig, source: str, times, amps, node: str) -> dict:
    """One row of batch_results.csv for a run's amplitude series, with the
    reference's fits and rounding (ymgpu2d/analysis/batch_analyze.py:213-238)."""
    d = derive(cfg)
    kz = cfg.k_mode * 2.0 * math.pi / d.lz
    gamma, t0, t1, r2 = growth.fit_growth_rate(times, amps)
    pl = growth.fit_growth_rate_plateau(times, amps)
    gex = growth.wkb_exact_gamma(d.alpha, d.V0, kz)

    def r1(v):
        return round(v, 1) if math.isfinite(v) else math.nan

    return {"kz": kz, "alpha": d.alpha, "V0": d.V0, "xi_sponge": cfg.xi_sponge,
            "gamma_sim": round(gamma, 5), "gamma_exact": round(gex, 5),
            "ratio": round(gamma / gex, 3) if gex > 0 else math.nan, "R2": round(r2, 4),
            "t0": r1(t0), "t1": r1(t1), "has_plateau": pl["has_plateau"],
            "gamma_plateau": round(pl["gamma"], 5) if math.isfinite(pl["gamma"]) else math.nan,
            "plateau_t0": r1(pl["t0"]), "plateau_t1": r1(pl["t1"]),
            "plateau_ratio": round(pl["gamma"] / gex, 3) if (gex > 0 and math.isfinite(pl["gamma"])) else math.nan,
            "source": source, "node": node}


@dataclass
class CampaignResult:
    run: CampaignRun
    out_dir: Path
    status: str = "pending"  # done | halted | rejected
    halt_reason: str = ""
    steps: int = 0
    times: list = field(default_factory=list)
    amps: list = field(default_factory=list)
    amps_conj: list = field(default_factory=list)
    row: dict | None = None
    seconds: float = math.nan


class CampaignRunner:
    """Runs a campaign's configurations together on one GPU.

    out_root: where each run's output directory goes.
    budget_bytes: device memory the resident runs may hold together.
    snapshots: None, "csv" (the reference's ym_%06d.csv) or "fp64", written
        at each export besides the amplitude.
    on_start: called as on_start(run) after a run's initial state is made
        and before its first energy (e.g. to add noise).
    seed_dir: directory that relative ``seed_profile_file`` paths are
        relative to (where the reference's script ran ym_coupled).
    node: the ``node`` column of batch_results.csv.
    """

    def __init__(self, out_root: str | Path, budget_bytes: int = 150 << 30, device="cuda", graph_steps: int = 4,
                 snapshots: str | None = None, on_start=None, seed_dir: str | Path | None = None, node: str = "b200"):
        self.out_root = Path(out_root)
        self.budget = int(budget_bytes)
        self.device = device
        self.graph_steps = graph_steps
        self.snapshots = snapshots
        self.on_start = on_start
        self.seed_dir = Path(seed_dir) if seed_dir is not None else None
        self.node = node

    def plan(self, runs: list) -> list:
        """(run, config, footprint bytes, total steps) per run; no GPU."""
        out = []
        for r in runs:
            cfg = loads(r.ini, r.name)
            d = derive(cfg)
            out.append((r, cfg, footprint(cfg), d.total_steps))
        return out

    def _start(self, r: CampaignRun, cfg: RunConfig, res: CampaignResult, stream):
        from .run import KHRun, RunLoop

        run = KHRun(cfg, device=self.device, graph_steps=self.graph_steps)
        seed = cfg.seed_profile_file or None
        if seed and self.seed_dir is not None and not Path(seed).is_absolute():
            seed = str(self.seed_dir / seed)
        run.init(seed_file=seed, stream=stream)
        if self.on_start:
            self.on_start(run)
        res.out_dir.mkdir(parents=True, exist_ok=True)

        def record(kr, step):
            a, ac = kr.circ_amp("Az", k=cfg.k_mode, stream=stream)
            res.times.append(step * kr.d.dt)
            res.amps.append(a)
            res.amps_conj.append(ac)

        loop = RunLoop(run, csv=res.out_dir / "energy.csv", stream=stream, on_export=record,
                       export_dir=res.out_dir if self.snapshots else None, export_format=self.snapshots or "csv")
        loop.start()
        return run, loop

    def _finish(self, res: CampaignResult, cfg: RunConfig, run, loop, t0: float):
        loop.close()
        res.status = "halted" if run.halted else "done"
        res.halt_reason = run.halt_reason
        res.steps = run.step_count
        res.seconds = time.perf_counter() - t0
        kz = cfg.k_mode * 2.0 * math.pi / run.d.lz
        with open(res.out_dir / f"timeseries_k{kz_label(kz)}.csv", "w", newline="") as fh:
            w = csv.writer(fh)
            w.writerow(["t", "amp", "amp_conj"])
            for row in zip(res.times, res.amps, res.amps_conj):
                w.writerow([repr(float(v)) for v in row])
        if len(res.times) >= 5:
            import numpy as np

            res.row = result_row(cfg, res.out_dir.name, np.array(res.times), np.array(res.amps), self.node)
        run.close()

    def run(self, runs: list) -> list:
        import torch

        from .batch import KHBatch

        stream = torch.cuda.Stream(device=self.device)
        batch = KHBatch(device=self.device, graph_steps=self.graph_steps)
        results = []
        pending = deque()
        for r, cfg, fp, _steps in self.plan(runs):
            res = CampaignResult(r, self.out_root / out_dir_name(cfg))
            results.append(res)
            if fp > self.budget:
                res.status = "rejected"
            else:
                pending.append((r, cfg, fp, res))
        active = []  # (res, cfg, run, loop, fp, t0)
        used = 0
        try:
            while pending or active:
                while pending and used + pending[0][2] <= self.budget:
                    r, cfg, fp, res = pending.popleft()
                    t0 = time.perf_counter()
                    run, loop = self._start(r, cfg, res, stream)
                    if loop.finished:  # nothing to step (zero steps)
                        self._finish(res, cfg, run, loop, t0)
                        continue
                    batch.add(run)
                    active.append((res, cfg, run, loop, fp, t0))
                    used += fp
                if not active:
                    continue
                n = min(a[3].steps_to_event() for a in active)
                batch.step(n, stream)
                keep = []
                for a in active:
                    res, cfg, run, loop, fp, t0 = a
                    loop.after_steps()
                    if loop.finished:
                        batch.remove(run)
                        self._finish(res, cfg, run, loop, t0)
                        used -= fp
                    else:
                        keep.append(a)
                active = keep
        finally:
            for res, cfg, run, loop, fp, t0 in active:
                loop.close()
                run.close()
            batch.close()
        self.write_results(results)
        return results

    def write_results(self, results: list) -> Path:
        """batch_results.csv of the runs with a fit, sorted by (alpha, V0, kz)
        as batch_analyze.py sorts it."""
        rows = sorted((r.row for r in results if r.row), key=lambda x: (x["alpha"], x["V0"], x["kz"]))
        self.out_root.mkdir(parents=True, exist_ok=True)
        path = self.out_root / "batch_results.csv"
        with open(path, "w", newline="") as fh:
            w = csv.DictWriter(fh, fieldnames=RESULT_COLUMNS)
            w.writeheader()
            w.writerows(rows)
        return path


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description="Run campaign shell scripts as one batched job on one GPU")
    ap.add_argument("scripts", nargs="+", help="campaign scripts (heredoc .ini + ym_coupled lines)")
    ap.add_argument("--out", required=True, help="output root (one directory per run, as ym_coupled names it)")
    ap.add_argument("--budget-gb", type=float, default=150.0)
    ap.add_argument("--snapshots", choices=["csv", "fp64"], default=None)
    ap.add_argument("--seed-dir", default=None, help="directory relative seed_profile_file paths start from")
    ap.add_argument("--dry-run", action="store_true", help="list the runs, footprints and steps; no GPU")
    args = ap.parse_args(argv)
    runs = []
    for s in args.scripts:
        runs += parse_campaign_script(Path(s).read_text())
    runner = CampaignRunner(args.out, int(args.budget_gb * (1 << 30)), snapshots=args.snapshots,
                            seed_dir=args.seed_dir)
    if args.dry_run:
        for r, cfg, fp, steps in runner.plan(runs):
            print(f"{r.order:4d} {r.name:40s} {out_dir_name(cfg):60s} {fp / 2**20:10.1f} MiB {steps:9d} steps")
        return 0
    for res in runner.run(runs):
        print(f"{res.run.name:40s} {res.status:8s} {res.steps:9d} steps {res.seconds:8.2f} s {res.halt_reason}")
    return 0


if __name__ == "__main__":  # pragma: no cover
    raise SystemExit(main())
