"""Campaign front-end on the GPU: every run of a batched campaign writes
the files its lone run writes, byte for byte.

Four runs of different grids (so different time steps, energy strides and
export strides) and one run with a NaN planted in its initial state (it
halts at its first energy check) go through one CampaignRunner with a
budget that admits three at a time.  Each run's energy.csv and
timeseries_k<kz>.csv must equal what KHRun.run writes for the same .ini
alone, and batch_results.csv must hold one row per run with enough
samples.
"""
import csv
import math

import numpy as np
import pytest

from kh_simulations_b200 import campaign
from kh_simulations_b200.config import loads, out_dir_name
from kh_simulations_b200.run import KHRun
from kh_simulations_b200.server import footprint

pytestmark = pytest.mark.gpu

BASE = ("alpha_YM = 1.0\nrun_mode = 6\nV0 = 0.05\neps_override = 1.0\nlx_override = 20\n"
        "courant_override = 0.4\nperturb_amp = 0.15\nnz_override = 32\ntarget_tu = 6\n")
GRIDS = {"g48": "nx_override = 48\nk_mode = 1\n", "g64": "nx_override = 64\nk_mode = 2\n",
         "g40": "nx_override = 40\nk_mode = 1\nsuppress_kz0 = 1\n", "g96": "nx_override = 96\nk_mode = 3\n",
         "nan": "nx_override = 48\nk_mode = 1\nrun_tag = nan\n"}


def _plant_nan(run):
    if run.cfg.run_tag == "nan":
        run.state[13, 3, 5] = math.nan  # px of beam A: the energy is NaN from the start


def test_campaign_matches_lone_runs(tmp_path):
    runs = [campaign.CampaignRun(name, BASE + extra, i) for i, (name, extra) in enumerate(GRIDS.items())]
    budget = 3 * max(footprint(loads(r.ini, r.name)) for r in runs)
    runner = campaign.CampaignRunner(tmp_path / "camp", budget_bytes=budget, on_start=_plant_nan)
    results = runner.run(runs)
    assert [r.status for r in results] == ["done", "done", "done", "done", "halted"]
    for res in results:
        cfg = loads(res.run.ini, res.run.name)
        assert res.out_dir.name == out_dir_name(cfg)
        lone = KHRun(cfg)
        lone.init()
        _plant_nan(lone)
        amps = []
        lone_dir = tmp_path / "lone" / res.run.name
        lone_dir.mkdir(parents=True)
        lone.run(csv=lone_dir / "energy.csv", on_export=lambda r, s: amps.append(r.circ_amp("Az")))
        assert (res.out_dir / "energy.csv").read_bytes() == (lone_dir / "energy.csv").read_bytes(), res.run.name
        assert res.steps == lone.step_count and (res.status == "halted") == lone.halted
        ts = list(csv.reader(open(res.out_dir / f"timeseries_k{campaign.kz_label(cfg.k_mode)}.csv")))
        assert ts[0] == ["t", "amp", "amp_conj"]
        got = np.array([[float(v) for v in row] for row in ts[1:]])
        ref = np.array([[s * lone.d.dt, a, c] for s, (a, c) in zip(range(0, 10 ** 9, lone.d.export_stride), amps)])
        assert got.shape == ref.shape and np.array_equal(got[:, 1:], ref[:, 1:], equal_nan=True), res.run.name
        np.testing.assert_allclose(got[:, 0], ref[:, 0], rtol=1e-15)
        lone.close()
    rows = list(csv.DictReader(open(tmp_path / "camp" / "batch_results.csv")))
    assert len(rows) == sum(len(r.times) >= 5 for r in results) >= 4
    assert tuple(rows[0]) == campaign.RESULT_COLUMNS
