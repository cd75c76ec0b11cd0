"""Host logic of the serving loop (no GPU): footprints, FIFO admission
under the memory budget, rejection of oversized requests, the seeded
request mix and the latency percentiles."""
import math
from collections import deque

import numpy as np

from kh_simulations_b200.config import loads
from kh_simulations_b200.server import KHRequest, KHServer, _censor, _percentiles, footprint, poisson_mix


def cfg(nz, nx, extra=""):
    return loads(f"nz_override = {nz}\nnx_override = {nx}\n{extra}")


def test_footprint_counts_two_buffers_and_filter_scratch():
    base = footprint(cfg(64, 128))
    assert base >= 2 * 24 * 8 * 64 * 128
    assert footprint(cfg(64, 128, "kz_keep_max = 21\n")) > base


def test_footprint_of_the_tensor_core_filter():
    """The TF32 engine holds hi/lo tile images of the 21 filtered arrays
    (G: 8 bytes per array cell, x padded to 128) and of the coefficients."""
    fp64 = footprint(cfg(1024, 2048, "kz_keep_max = 341\n"))
    tf32 = footprint(cfg(1024, 2048, "kz_keep_max = 341\nfilter_engine = tf32x3\n"))
    g_images = 2 * 21 * 2048 * 1024 * 4
    assert tf32 - fp64 > g_images - 21 * 342 * 2048 * 8
    assert tf32 > 2 * 24 * 8 * 1024 * 2048 + g_images


def test_fifo_admission_respects_budget_and_rejects_oversize():
    small, big = cfg(32, 64), cfg(256, 512)
    budget = 3 * footprint(small)
    srv = KHServer(budget_bytes=budget)
    pend = deque([KHRequest(0, small, 10, 0.0), KHRequest(1, big, 10, 0.0), KHRequest(2, small, 10, 0.0),
                  KHRequest(3, small, 10, 5.0)])
    adm = srv.admit_order(pend, now=1.0, used=0)
    # the oversized request is rejected, the others admitted in order; the
    # not-yet-arrived one waits
    assert [r.rid for r, _ in adm] == [0, 2]
    assert [r.rid for r in pend] == [3]
    adm = srv.admit_order(pend, now=6.0, used=2 * footprint(small))
    assert [r.rid for r, _ in adm] == [3]


def test_head_of_line_blocks_when_budget_full():
    small = cfg(32, 64)
    srv = KHServer(budget_bytes=2 * footprint(small))
    pend = deque([KHRequest(i, small, 10, 0.0) for i in range(4)])
    adm = srv.admit_order(pend, now=0.0, used=footprint(small))
    assert [r.rid for r, _ in adm] == [0]
    assert len(pend) == 3


def test_poisson_mix_is_seeded_and_cfl_safe():
    a = poisson_mix(3, rate=20, duration=2.0, min_cells=128 * 256, max_cells=1024 * 2048, min_steps=50,
                    max_steps=200, base_ini="alpha_YM = 1.0\nlx_override = 20\n")
    b = poisson_mix(3, rate=20, duration=2.0, min_cells=128 * 256, max_cells=1024 * 2048, min_steps=50,
                    max_steps=200, base_ini="alpha_YM = 1.0\nlx_override = 20\n")
    assert [r.arrival for r in a] == [r.arrival for r in b]
    assert 10 <= len(a) <= 80
    from kh_simulations_b200.config import derive

    for r in a:
        d = derive(r.cfg)
        assert d.nx == 2 * d.nz
        assert d.dt * math.sqrt(d.dx ** -2 + d.dz ** -2) <= 0.4 + 1e-6
        if r.cfg.suppress_kz0:
            assert d.nz & (d.nz - 1) == 0


def test_percentiles():
    reqs = [KHRequest(i, cfg(32, 64), 1, arrival=0.0) for i in range(5)]
    for i, r in enumerate(reqs):
        r.finished, r.status = float(i + 1), "done"
    p50, p99 = _percentiles(reqs)
    assert p50 == 3.0 and abs(p99 - np.percentile([1, 2, 3, 4, 5], 99)) < 1e-12


def test_censoring_at_a_deadline():
    """Requests that arrived by the deadline but did not finish are
    'unfinished' with their latency censored at the deadline (the
    percentiles are then lower bounds); later arrivals are left out."""
    reqs = [KHRequest(i, cfg(32, 64), 1, arrival=float(i)) for i in range(4)]
    reqs[0].status, reqs[0].finished = "done", 0.5
    reqs[1].status = "running"
    _censor(reqs, end=2.5)
    assert [r.status for r in reqs] == ["done", "unfinished", "unfinished", "pending"]
    assert reqs[1].latency == 1.5 and reqs[2].latency == 0.5
    p50, _ = _percentiles(reqs)
    assert p50 == 0.5
