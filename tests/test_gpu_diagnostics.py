"""Device diagnostics and snapshots against the CPU restatements of the
reference's analysis scripts and CSV writer (oracle/diagnostics.py).

- ymkh_circ_amp: every colour-2/3 pair, x-mean and sech-weighted, within
  1e-12 of numpy's rfft amplitudes (plus 1e-13 of the summed terms' size,
  for amplitudes that cancel to rounding level); ymkh_mode_amp is its Az
  pair bit for bit.
- ymkh_gauss: the 16 root-mean-squares within 1e-12 of gauss_check.py's
  formulas (summation order differs: compensated on the device, pairwise in
  numpy; each cell's terms are evaluated operand for operand alike).
- ymkh_snapshot: the CSV is byte-identical to main_ym.cu's writer restated
  with printf "%g"; the FP64 form round-trips bit for bit; snapshots
  queued between steps hold the state of their own step.
"""
import math

import numpy as np
import pytest
import torch

from kh_simulations_b200 import growth, snapshot
from kh_simulations_b200._lib import YMKHError
from kh_simulations_b200.run import KHRun
from oracle import diagnostics as od

from cases import config

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def stepped_run():
    run = KHRun(config("ref_bands_kz0"))
    run.init()
    run.add_noise(1e-4, seed=3)
    run.step(7)
    yield run
    run.close()


@pytest.mark.parametrize("pair", ["Az", "By", "Ex", "Ez"])
@pytest.mark.parametrize("weighted", [False, True])
def test_circ_amp_matches_rfft(stepped_run, pair, weighted):
    run = stepped_run
    st = run.state_numpy()
    w = growth.xi_weight(run.d.nx, run.d.dx, eps=run.d.eps, lx=run.d.lx) if weighted else None
    re, im = st[od.IDX[pair + "2"]], st[od.IDX[pair + "3"]]
    # size of the terms summed: a removed z-mean leaves k = 0 at rounding level
    col = (np.abs(re).sum(axis=0) + np.abs(im).sum(axis=0)) / run.d.nz
    scale = float(col.mean() if w is None else np.dot(col, w))
    for k in (0, 1, 3):
        got = run.circ_amp(pair, k=k, weight=w)
        ref = od.circ_amp(re, im, k, w)
        for g, r in zip(got, ref):
            assert abs(g - r) <= 1e-12 * abs(r) + 1e-13 * scale, (pair, k, g, r, scale)


def test_mode_amp_is_the_az_pair(stepped_run):
    assert stepped_run.mode_amp(k=1) == stepped_run.circ_amp("Az", k=1)


def test_gauss_matches_gauss_check(stepped_run):
    run = stepped_run
    st = run.state_numpy()
    ref = od.gauss_terms(st, run.d.dx, run.d.dz, run.d.alpha)
    g = run.gauss()
    got = np.concatenate([g["G"], g["div_E"], g["nonabelian"], g["rho"], g["lhs"], [(g["Etot_scale"] - 1e-30) * run.d.dx]])
    assert ref[:3].min() > 0  # a residual to compare; exact zeros (e.g. rho^2 with Q2 = 0) must match exactly
    np.testing.assert_allclose(got, ref, rtol=1e-12, atol=0)


def test_snapshot_csv_bytes_and_fp64_round_trip(stepped_run, tmp_path):
    run = stepped_run
    st = run.state_numpy()
    run.snapshot(tmp_path / "s.csv", "csv")
    run.snapshot(tmp_path / "s.fp64", "fp64")
    run.snapshot_wait()
    assert (tmp_path / "s.csv").read_text() == od.snapshot_csv_text(st, run.d.dx, run.d.dz)
    back, dx, dz = snapshot.read_fp64(tmp_path / "s.fp64")
    assert (dx, dz) == (run.d.dx, run.d.dz)
    assert np.array_equal(back.view(np.uint64), st.view(np.uint64))
    cols = snapshot.read_csv(tmp_path / "s.csv")
    assert cols["By2"].shape == (run.d.nz, run.d.nx)
    np.testing.assert_allclose(cols["Az2"], st[od.IDX["Az2"]], rtol=1e-5, atol=1e-300)


def test_queued_snapshots_hold_their_own_step(tmp_path):
    """Six snapshots enqueued between steps without waiting (more than the
    four writers kept at once): each file holds the state of its step."""
    run = KHRun(config("no_filter"))
    run.init()
    states = []
    for k in range(6):
        run.snapshot(tmp_path / f"q{k}.fp64", "fp64")
        states.append(run.state.clone())  # same stream: ordered after the snapshot copies
        run.step(3)
    run.snapshot_wait()
    for k in range(6):
        back, _, _ = snapshot.read_fp64(tmp_path / f"q{k}.fp64")
        assert np.array_equal(back, states[k].cpu().numpy()), k
    run.close()


def test_snapshot_write_error_is_reported(tmp_path):
    run = KHRun(config("no_filter"))
    run.init()
    run.snapshot(tmp_path / "missing_dir" / "x.csv", "csv")
    with pytest.raises(YMKHError, match="cannot open"):
        run.snapshot_wait()
    run.snapshot_wait()  # the error is reported once
    run.close()


def test_run_exports_at_the_reference_stride(tmp_path):
    """ym_%06d files at step 0 and every export stride, after the energy
    check of the same step (main_ym.cu:457-477)."""
    run = KHRun(config("no_filter"))
    run.init()
    seen = []
    run.run(total_steps=25, energy_stride=4, export_dir=tmp_path, export_format="csv", export_stride=10,
            on_export=lambda r, s: seen.append((s, r.step_count, len(r.history))))
    names = sorted(p.name for p in tmp_path.iterdir())
    assert names == ["ym_000000.csv", "ym_000010.csv", "ym_000020.csv"]
    assert [s for s, _, _ in seen] == [0, 10, 20]
    assert all(s == c for s, c, _ in seen)
    # the energy records of steps 0, 4, 8 exist when step 10 is exported
    assert seen[1][2] == 3
    st = snapshot.read_csv(tmp_path / "ym_000020.csv")
    assert st["nA"].shape == (run.d.nz, run.d.nx)
    assert math.isfinite(float(st["nA"].sum()))
    run.close()


def test_circ_amp_rejects_bad_arguments(stepped_run):
    with pytest.raises(ValueError):
        stepped_run.circ_amp("By", weight=np.ones(3))
    out = (__import__("ctypes").c_double * 2)()
    rc = stepped_run.lib.ymkh_circ_amp(stepped_run.ctx, 9, 1, None, out, None)
    assert rc != 0
    torch.cuda.synchronize()
