"""Shared parity cases: small .ini configurations covering every stage of the
step (filters, z-mean, sponge, xi_cut, hyperdiffusion, warm closure, wall
boundaries, every run_mode of the initial state)."""
from __future__ import annotations

from kh_simulations_b200.config import loads

# The configuration the headline workload scales up: alpha=1, V0=0.05,
# shear width 1, kz=1 seed of amplitude 0.15*V0, Lx=20 (shear), Lz=2pi,
# CFL 0.4, modes above NZ/3 subtracted.
BASE = """
k_mode = 1
alpha_YM = 1.0
perturb_amp = 0.15
run_mode = 6
V0 = 0.05
eps_override = 1.0
lx_override = 20
courant_override = 0.4
"""

CASES = {
    # NZ x NX small enough for the CPU oracle; NZ % 32 == 0 for the bands
    "keep_third": BASE + "nz_override = 32\nnx_override = 48\nkz_keep_max = 10\n",
    "no_filter": BASE + "nz_override = 32\nnx_override = 48\n",
    "ref_bands_kz0": BASE + "nz_override = 32\nnx_override = 48\nsuppress_kz0 = 1\nkz_suppress_max = 2\nkz_suppress_hi = 9\n",
    "sponge_cut": BASE + "nz_override = 32\nnx_override = 48\nxi_sponge = 6\nsigma_sponge = 5\nxi_cut = 8\n",
    # the reference updates in place while neighbours read (a race it
    # documents); the CUDA path and the oracle both use the race-free form
    "hyperdiff": BASE + "nz_override = 32\nnx_override = 48\nhyp_diff = 5e-5\n",
    "warm": BASE + "nz_override = 32\nnx_override = 48\nwarm_T = 0.01\n",
    "wall_mode0": BASE.replace("run_mode = 6", "run_mode = 0") + "nz_override = 32\nnx_override = 48\n",
    "dtanh_mode3": BASE.replace("run_mode = 6", "run_mode = 3") + "nz_override = 32\nnx_override = 48\n",
    "step_mode4": BASE.replace("run_mode = 6", "run_mode = 4") + "nz_override = 32\nnx_override = 40\n",
    "cos_mode5": BASE.replace("run_mode = 6", "run_mode = 5") + "nz_override = 32\nnx_override = 48\n",
    "circ_mode1": BASE.replace("run_mode = 6", "run_mode = 1") + "nz_override = 32\nnx_override = 48\n",
    "emhd_mode2": BASE.replace("run_mode = 6", "run_mode = 2") + "nz_override = 32\nnx_override = 48\n",
    "taper_by1eq": BASE + "nz_override = 32\nnx_override = 48\nvz_edge_taper = 4\ninit_by1_eq = 1\n",
    "unfrozen": BASE + "nz_override = 32\nnx_override = 48\nfreeze_override = 0\n",
    # ragged sizes: NX not a multiple of any strip width, odd NZ
    "ragged": BASE + "nz_override = 27\nnx_override = 37\n",
}

# Cases whose step has no band filter: bit-identical to the reference.
BITWISE = {"no_filter", "sponge_cut", "warm", "wall_mode0", "dtanh_mode3", "step_mode4", "cos_mode5",
           "circ_mode1", "emhd_mode2", "taper_by1eq", "unfrozen", "ragged"}


def config(name: str):
    return loads(CASES[name], name)


# Cases stored as golden vectors from the reference's own kernels (32 x 32
# grids keep the fixtures small).
GOLDEN = ("keep_third", "ref_bands_kz0", "no_filter", "wall_mode0", "sponge_cut", "warm", "dtanh_mode3",
          "step_mode4", "cos_mode5", "circ_mode1", "emhd_mode2", "taper_by1eq", "unfrozen", "ragged")
GOLDEN_STEPS = 2


def golden_config(name: str):
    text = CASES[name].replace("nx_override = 48", "nx_override = 32")
    return loads(text, name)
