"""CPU restatements of the reference's offline diagnostics — TEST
INFRASTRUCTURE ONLY (the checker for ymkh_circ_amp, ymkh_gauss and
ymkh_snapshot; never the product path).

The reference computes these in its analysis scripts from 6-digit CSV
snapshots; here they take the FP64 state ([24, NZ, NX], include/ymkh.h
order) so that the device results can be compared at FP64 precision.

- circ_amp: ymgpu2d/analysis/remote_timeseries.py:62-77 (x-mean) and
  ymgpu2d/analysis/resolution_convergence.py:77-86 (sech-weighted).
- gauss_terms: ymgpu2d/analysis/gauss_check.py:40-110, with the state's own
  Az1 in place of the script's reconstructed background (it rebuilds Az1
  only because snapshots older than the 26-column format lack it).
- snapshot_csv_text: the CSV writer of ymgpu2d/main_ym.cu:287-306.

Parity pinned: the growth-rate fitters fed by these amplitudes are checked
against the reference's own outputs (tests/golden/growth_fits.json); the
CSV layout follows the writer's source line for line.
"""
from __future__ import annotations

import numpy as np

NAMES = ("Ex1", "Ex2", "Ex3", "Ez1", "Ez2", "Ez3", "By1", "By2", "By3", "Az1", "Az2", "Az3",
         "nA", "pxA", "pzA", "Q1A", "Q2A", "Q3A", "nB", "pxB", "pzB", "Q1B", "Q2B", "Q3B")
IDX = {n: i for i, n in enumerate(NAMES)}

CSV_COLUMNS = ("X", "Z", "By1", "By2", "By3", "Az2", "Az3", "PzA", "PxA", "Q1A", "PzB", "PxB", "Q1B",
               "Ex1", "Ex2", "Ex3", "Ez1", "Ez2", "Ez3", "nA", "nB", "Q2A", "Q3A", "Q2B", "Q3B", "Az1")
# CSV column -> state array
_CSV_SRC = {"PzA": "pzA", "PxA": "pxA", "PzB": "pzB", "PxB": "pxB"}


def circ_amp(re: np.ndarray, im: np.ndarray, k: int, weight: np.ndarray | None = None) -> tuple:
    """(|F2 + i F3|, |F2 - i F3|) at wavenumber k along z (axis 0), averaged
    over x: the mean / NZ (remote_timeseries.py:70-74) or, with a weight,
    sum_x w |rfft/NZ| (resolution_convergence.py:83-86)."""
    nz = re.shape[0]
    fre = np.fft.rfft(re, axis=0)[k, :] / nz
    fim = np.fft.rfft(im, axis=0)[k, :] / nz
    amp, amp_c = np.abs(fre + 1j * fim), np.abs(fre - 1j * fim)
    if weight is None:
        return float(amp.mean()), float(amp_c.mean())
    return float(np.dot(amp, weight)), float(np.dot(amp_c, weight))


def gauss_terms(st: np.ndarray, dx: float, dz: float, alpha: float) -> np.ndarray:
    """The 16 root-mean-squares of ymkh_gauss: G^a, div E^a, alpha (Az x Ez)^a,
    rho^a, div E^a + alpha (Az x Ez)^a (a = 1..3), |Ex1|+..+|Ez3|."""
    f = {n: st[IDX[n]] for n in NAMES}
    rms = lambda a: np.sqrt(np.mean(a ** 2))  # noqa: E731

    def div_e(ex, ez):
        return (ex - np.roll(ex, 1, axis=1)) / dx + (ez - np.roll(ez, 1, axis=0)) / dz

    def centre_z(ez):
        return 0.5 * (ez + np.roll(ez, 1, axis=0))

    de = [div_e(f[f"Ex{a}"], f[f"Ez{a}"]) for a in (1, 2, 3)]
    ezc = [centre_z(f[f"Ez{a}"]) for a in (1, 2, 3)]
    az1, az2, az3 = f["Az1"], f["Az2"], f["Az3"]
    nab = [alpha * (az2 * ezc[2] - az3 * ezc[1]),
           alpha * (az3 * ezc[0] - az1 * ezc[2]),
           alpha * (az1 * ezc[1] - az2 * ezc[0])]
    rho = [f[f"Q{a}A"] * f["nA"] + f[f"Q{a}B"] * f["nB"] for a in (1, 2, 3)]
    g = [de[a] + nab[a] - rho[a] for a in range(3)]
    lhs = [de[a] + nab[a] for a in range(3)]
    all_e = (np.abs(f["Ex1"]) + np.abs(f["Ex2"]) + np.abs(f["Ex3"])
             + np.abs(f["Ez1"]) + np.abs(f["Ez2"]) + np.abs(f["Ez3"]))
    return np.array([rms(v) for v in (*g, *de, *nab, *rho, *lhs, all_e)])


def snapshot_csv_text(st: np.ndarray, dx: float, dz: float) -> str:
    """The 26-column snapshot of main_ym.cu:287-306: X = x*DX, Z = z*DZ and
    the arrays, each printed as an ostream of default precision prints a
    double (printf "%g"), rows z-major with x fastest."""
    nz, nx = st.shape[1:]
    cols = [st[IDX[_CSV_SRC.get(c, c)]].reshape(-1) for c in CSV_COLUMNS[2:]]
    out = [",".join(CSV_COLUMNS) + "\n"]
    for z in range(nz):
        for x in range(nx):
            i = x + z * nx
            out.append(",".join(["%g" % (x * dx), "%g" % (z * dz)] + ["%g" % c[i] for c in cols]) + "\n")
    return "".join(out)
