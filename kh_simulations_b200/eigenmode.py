"""Eigenmode seeds: the linear Kelvin–Helmholtz mode of the NAB_CIRC
background, solved in-process so that a run can start from it without the
reference's offline step.

The reference solves it with ymgpu2d/analysis/ym_eigenmode.py and writes
``seeds/eigenmode_seed_*.bin`` for ``seed_profile_file``:
- the complex colour-2 + i colour-3 fields (b, ex, ez, a, qA, qB) linearised
  about Az1 = -V0 log cosh(xi), vz = +-V0 tanh(xi), xi = (x - LX/2)/EPS,
  with d/dt -> gamma and d/dz -> i kz, on the periodic x grid of the
  simulation's staggering (forward difference for dEz/dx in Faraday,
  backward for dB/dx in Ampere; ym_eigenmode.py:89-198), plus the sponge
  damping sigma_sponge (|xi| - xi_sponge) where |xi| > xi_sponge, or a
  hard wall beyond xi_cut;
- the 10 eigenvalues nearest the shift 0.55 gamma_WKB (0.1 without a WKB
  root), by ARPACK in shift-invert mode (:201-232);
- of those, the one with the largest real part above 1e-5 (of a pair with
  equal real parts, the one with positive imaginary part) whose |b| peaks
  inside 1.15 xi_inner and is below 15% of its peak at both ends of the
  box, else the first growing one (:244-258, :349-372);
- the six profiles rotated so that a is real and positive at its largest
  modulus, divided by that modulus, and their real parts stored as float32
  (:411-440).

Here the operator is assembled from whole-array blocks rather than entry
by entry, and ``solve_many`` spreads many parameter points over worker
processes.  The profiles are the reference's to float32 rounding
(tests/test_eigenmode.py).
"""
from __future__ import annotations

import functools
import math
from dataclasses import dataclass

import numpy as np

from .seed import FIELD_ORDER

NX_DEFAULT = 384  # the reference solver's default grid (ym_eigenmode.py:55)


@dataclass(frozen=True)
class ModeSpec:
    """One eigenmode problem. kz is the integer mode number k_mode; the
    physical wavenumber is k_mode * 2 pi / lz."""
    k_mode: int
    alpha: float
    V0: float
    eps: float = 0.15
    nx: int = NX_DEFAULT
    lx: float = 6.0 * math.pi
    lz: float = 2.0 * math.pi
    xi_sponge: float = 10.0  # 0: no sponge
    sigma_sponge: float = 5.0
    xi_cut: float | None = None
    shift: float | None = None  # None: 0.55 gamma_WKB

    @property
    def kz(self) -> float:
        return self.k_mode * 2.0 * math.pi / self.lz


@dataclass
class Mode:
    spec: ModeSpec
    gamma: complex
    gamma_wkb: float
    localised: bool
    fields: dict   # complex profiles b, ex, ez, a, qA, qB (length nx)
    eigenvalues: np.ndarray

    def seed_profiles(self) -> dict:
        """{by, ex, ez, az, qA, qB}: float32 real parts after the rotation and
        scaling of the reference's seed export."""
        a = self.fields["a"]
        i = int(np.argmax(np.abs(a)))
        rot = np.exp(-1j * np.angle(a[i]))
        scale = np.max(np.abs(a))
        names = ("b", "ex", "ez", "a", "qA", "qB")
        return {out: ((self.fields[src] * rot).real / scale).astype(np.float32)
                for out, src in zip(FIELD_ORDER, names)}


def wkb_gamma(kz: float, alpha: float, V0: float, n: int = 0) -> float:
    """Im(omega) of the fastest root of omega^4 - kz^2 omega^2
    - (2n+1) sqrt(alpha^3/2) V0 omega - alpha^2 V0 kz = 0, NaN when no root
    grows (ym_eigenmode.py:58-84)."""
    if alpha == 0:
        return math.nan
    c = (2 * n + 1) * math.sqrt(alpha ** 3 / 2.0) * V0
    roots = np.roots([1.0, 0.0, -kz ** 2, -c, -alpha ** 2 * V0 * kz])
    grow = roots[roots.imag > 1e-10]
    return float(np.max(grow.imag)) if len(grow) else math.nan


def operator(spec: ModeSpec):
    """The 6N x 6N complex sparse operator L (gamma psi = L psi), state order
    [b, ex, ez, a, qA, qB], as CSR."""
    import scipy.sparse as sp

    n = spec.nx
    dx = spec.lx / n
    x = np.arange(n) * dx
    xi = (x - spec.lx / 2.0) / spec.eps
    az1 = -spec.V0 * np.log(np.cosh(xi))
    vz = spec.V0 * np.tanh(xi)
    om_a = spec.kz + spec.alpha * az1
    om_f = spec.kz - spec.alpha * az1
    i = np.arange(n)
    ip, im = (i + 1) % n, (i - 1) % n
    B, EX, EZ, A, QA, QB = (k * n for k in range(6))
    inside = np.ones(n, bool) if spec.xi_cut is None else np.abs(xi) <= spec.xi_cut
    ok_p, ok_m = inside[ip], inside[im]
    rows, cols, vals = [], [], []

    def put(r, c, v, mask=None):
        v = np.broadcast_to(np.asarray(v, dtype=complex), r.shape)
        if mask is not None:
            r, c, v = r[mask], c[mask], v[mask]
        rows.append(r)
        cols.append(c)
        vals.append(v)

    ii = i[inside]
    sel = lambda arr: arr[inside]  # noqa: E731
    # Faraday: gamma b = -i om_f ex + (ez[i+1] - ez[i]) / dx
    put(B + ii, EX + ii, -1j * sel(om_f))
    put(B + ii, EZ + ii, -1.0 / dx)
    put(B + ii, EZ + sel(ip), 1.0 / dx, sel(ok_p))
    # Ampere x: gamma ex = -i om_a b
    put(EX + ii, B + ii, -1j * sel(om_a))
    # Ampere z: gamma ez = (b[i] - b[i-1]) / dx + vz qA - vz qB
    put(EZ + ii, B + ii, 1.0 / dx)
    put(EZ + ii, B + sel(im), -1.0 / dx, sel(ok_m))
    put(EZ + ii, QA + ii, sel(vz))
    put(EZ + ii, QB + ii, -sel(vz))
    # potential: gamma a = -ez
    put(A + ii, EZ + ii, -1.0)
    # precession (Doppler-shifted): gamma qA = i alpha vz a - i vz om_a qA; qB with +i vz om_a
    put(QA + ii, A + ii, 1j * spec.alpha * sel(vz))
    put(QA + ii, QA + ii, -1j * sel(vz) * sel(om_a))
    put(QB + ii, A + ii, 1j * spec.alpha * sel(vz))
    put(QB + ii, QB + ii, 1j * sel(vz) * sel(om_a))
    # hard wall: the rows outside xi_cut hold explicit zeros
    out = i[~inside]
    for blk in range(6):
        put(blk * n + out, blk * n + out, 0.0)
    # sponge on every block's diagonal
    if spec.xi_sponge > 0:
        excess = np.abs(xi) - spec.xi_sponge
        damp = i[excess > 0]
        for blk in range(6):
            put(blk * n + damp, blk * n + damp, -spec.sigma_sponge * excess[excess > 0])
    L = sp.coo_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(6 * n, 6 * n))
    return L.tocsr()


def _localised(b: np.ndarray, spec: ModeSpec, xi_inner: float, frac: float = 0.15) -> bool:
    amp = np.abs(b)
    ip = int(np.argmax(amp))
    xi_peak = abs(ip * spec.lx / spec.nx - spec.lx / 2.0) / spec.eps
    return xi_peak < 1.15 * xi_inner and max(amp[0], amp[-1]) < frac * amp[ip]


def solve(spec: ModeSpec, n_eigs: int = 10) -> Mode | None:
    """The dominant localised growing mode of ``spec``, or None when no
    eigenvalue near the shift grows."""
    import scipy.sparse.linalg as spla

    L = operator(spec)
    gw = wkb_gamma(spec.kz, spec.alpha, spec.V0)
    shift = spec.shift
    if shift is None:
        shift = 0.55 * gw if (math.isfinite(gw) and gw > 0) else 0.1
    try:
        vals, vecs = spla.eigs(L, k=n_eigs, sigma=shift, which="LM", maxiter=10000, tol=1e-10)
    except spla.ArpackNoConvergence as e:
        vals, vecs = e.eigenvalues, e.eigenvectors
        if len(vals) == 0:
            return None
    # largest real part first; members of a pair whose real parts agree to
    # 12 digits in the order of their imaginary parts, positive first (the
    # reference leaves such a pair in ARPACK's order)
    order = np.lexsort((-vals.imag, -np.round(vals.real, 12)))
    vals, vecs = vals[order], vecs[:, order]
    n = spec.nx
    xi_inner = spec.xi_sponge if spec.xi_sponge > 0 else 5.0
    pick = next((j for j, v in enumerate(vals) if v.real >= 1e-5 and _localised(vecs[:n, j], spec, xi_inner)), None)
    if pick is None:
        pick = next((j for j, v in enumerate(vals) if v.real > 1e-5), None)
    if pick is None:
        return None
    v = vecs[:, pick]
    fields = {k: v[m * n:(m + 1) * n] for m, k in enumerate(("b", "ex", "ez", "a", "qA", "qB"))}
    return Mode(spec, complex(vals[pick]), gw, _localised(fields["b"], spec, xi_inner), fields, vals)


@functools.lru_cache(maxsize=64)
def cached_seed(spec: ModeSpec) -> dict:
    """Seed profiles of ``spec``, solved once per process per problem (runs of
    one campaign often share one)."""
    m = solve(spec)
    if m is None:
        raise ValueError(f"no growing eigenmode for {spec}")
    return m.seed_profiles()


def _solve_profiles(spec: ModeSpec):
    m = solve(spec)
    return None if m is None else (m.gamma, m.seed_profiles())


def solve_many(specs: list, workers: int = 0) -> list:
    """(gamma, seed profiles) or None per spec; with workers > 1 the points
    are spread over that many processes (started with spawn, so that a CUDA
    context in this process is never forked)."""
    if workers <= 1 or len(specs) <= 1:
        return [_solve_profiles(s) for s in specs]
    import multiprocessing as mp
    from concurrent.futures import ProcessPoolExecutor

    with ProcessPoolExecutor(max_workers=workers, mp_context=mp.get_context("spawn")) as ex:
        return list(ex.map(_solve_profiles, specs))


def seed_file_name(spec: ModeSpec) -> str:
    """The file name the reference's solver gives the seed
    (ym_eigenmode.py:420-433)."""
    lz_tag = f"_lz{spec.lz:.4f}" if abs(spec.lz - 2.0 * math.pi) > 1e-6 else ""
    lx_tag = f"_lx{spec.lx:.4f}" if abs(spec.lx - 6.0 * math.pi) > 1e-6 else ""
    eps_tag = f"_EPS{spec.eps:.3f}" if abs(spec.eps - 0.15) > 1e-6 else ""
    return (f"eigenmode_seed_kz{spec.k_mode}_a{spec.alpha:.2f}_V{spec.V0:.3f}{eps_tag}"
            f"_sp{spec.xi_sponge:.1f}{lz_tag}{lx_tag}.bin")


def _decimal(x: float) -> float:
    """The shortest decimal of a float32 value (0.05 for the float32 0.05 an
    .ini holds), as the reference's solver is given it on its command line;
    other values unchanged."""
    f = np.float32(x)
    return float(str(f)) if float(f) == x else x


def spec_for_run(cfg, d=None, nx: int = NX_DEFAULT) -> ModeSpec:
    """The eigenmode problem of a run's parameters, on the solver's own grid
    of ``nx`` points (the seed is interpolated to the run's grid as a seed
    file is).  Parameters that the .ini holds as float32 are passed as their
    shortest decimals, as the reference's campaign tools pass them."""
    from .config import derive

    d = d or derive(cfg)
    return ModeSpec(k_mode=cfg.k_mode, alpha=_decimal(d.alpha), V0=_decimal(d.V0), eps=_decimal(d.eps), nx=nx,
                    lx=_decimal(d.lx), lz=_decimal(d.lz), xi_sponge=_decimal(cfg.xi_sponge),
                    sigma_sponge=_decimal(cfg.sigma_sponge) if cfg.xi_sponge > 0 else 5.0)
