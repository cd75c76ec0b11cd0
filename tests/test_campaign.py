"""Campaign front-end, host side (CPU): reading campaign shell scripts,
planning, the result rows."""
import math

import numpy as np

from kh_simulations_b200 import campaign
from kh_simulations_b200.config import derive, loads, out_dir_name

# A script in the form ymgpu2d/analysis/gen_*_campaign.py writes
# (heredoc .ini, then ym_coupled on it), with the variants the reader
# must handle: quoted and bare heredoc tags, an .ini written twice, an
# .ini never run, comments and a subshell.
SCRIPT = """#!/bin/bash
set -e
# campaign: two alphas
cat > /tmp/run_a1.ini <<'EOINI'
k_mode = 1
alpha_YM = 1.0
V0 = 0.05
nz_override = 32
nx_override = 48
target_tu = 6
EOINI
echo "start a1"
cd /data/ymgpu2d && ./ym_coupled /tmp/run_a1.ini
cat > /tmp/unused.ini <<ENDINI
k_mode = 9
ENDINI
cat > /tmp/run_a2.ini <<"END"
k_mode = 2
alpha_YM = 2.0
END
cat > /tmp/run_a2.ini <<'EOINI'
  k_mode = 3
  alpha_YM = 2.5
  nz_override = 64
  nx_override = 96
EOINI
(cd /data/ymgpu2d/outputs && /data/ymgpu2d/ym_coupled /tmp/run_a2.ini >> log 2>&1) || echo "CRASHED"
# ./ym_coupled /tmp/unused.ini   (commented out)
"""


def test_parse_campaign_script():
    runs = campaign.parse_campaign_script(SCRIPT)
    assert [r.name for r in runs] == ["run_a1", "run_a2"]
    assert [r.order for r in runs] == [0, 1]
    c1 = loads(runs[0].ini, "a1")
    assert (c1.k_mode, c1.alpha_YM, c1.nz_override, c1.nx_override, c1.target_tu) == (1, 1.0, 32, 48, 6.0)
    c2 = loads(runs[1].ini, "a2")  # the text written last before the run
    assert (c2.k_mode, c2.alpha_YM, c2.nz_override) == (3, 2.5, 64)


def test_kz_label():
    got = [campaign.kz_label(k) for k in (1, 2.0, 1.5, 0.125, 0.25, 3.375)]
    assert got == ["1", "2", "1p5", "0p125", "0p25", "3p375"]


def test_plan_and_dry_run(tmp_path, capsys):
    path = tmp_path / "c.sh"
    path.write_text(SCRIPT)
    assert campaign.main([str(path), "--out", str(tmp_path / "out"), "--dry-run"]) == 0
    out = capsys.readouterr().out.splitlines()
    first = loads(campaign.parse_campaign_script(SCRIPT)[0].ini, "a1")
    assert len(out) == 2 and "run_a1" in out[0] and out_dir_name(first) in out[0]
    runner = campaign.CampaignRunner(tmp_path, budget_bytes=1 << 30)
    plan = runner.plan(campaign.parse_campaign_script(SCRIPT))
    assert plan[0][3] == derive(plan[0][1]).total_steps
    assert plan[1][2] > plan[0][2]  # a larger grid holds more memory


def test_result_row_uses_the_reference_fits_and_rounding():
    cfg = loads("k_mode = 2\nalpha_YM = 1.0\nV0 = 0.05\nxi_sponge = 10\n", "r")
    t = np.arange(0.0, 40.0, 1.0)
    a = 1e-9 * np.exp(0.0712345678 * t)
    row = campaign.result_row(cfg, "ym_src", t, a, "b200")
    assert tuple(row) == campaign.RESULT_COLUMNS
    assert row["kz"] == 2.0 and row["gamma_sim"] == round(0.0712345678, 5)
    assert row["R2"] == 1.0 and row["has_plateau"]
    assert row["gamma_exact"] > 0 and row["ratio"] == round(row["gamma_sim"] / row["gamma_exact"], 3)
    assert row["source"] == "ym_src" and math.isfinite(row["t0"])


def test_runs_over_budget_are_planned_as_such(tmp_path):
    runner = campaign.CampaignRunner(tmp_path, budget_bytes=1024)
    plan = runner.plan(campaign.parse_campaign_script(SCRIPT))
    assert all(fp > 1024 for _, _, fp, _ in plan)
