"""Batched and served forms give the same results as the plain step.

A run advanced inside a batch (one fused FCT and one fused Maxwell launch
over the tiles of every member) must be bit-identical to the same run
advanced alone, including when members join and leave between calls
(continuous batching), and the serving loop's results must equal the same
requests run one by one."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MIX = [
    ("nz_override = 64\nnx_override = 128\nkz_keep_max = 21\n", 0),
    ("nz_override = 32\nnx_override = 96\nsuppress_kz0 = 1\n", 1),
    ("nz_override = 128\nnx_override = 256\nhyp_diff = 5e-5\nkz_suppress_hi = 9\n", 2),
    ("nz_override = 27\nnx_override = 37\n", 3),        # ragged sizes: element load path
    ("nz_override = 32\nnx_override = 48\nrun_mode = 0\n", 0),  # walls
]


def _cfg(text):
    from cases import BASE
    from kh_simulations_b200.config import loads

    return loads(BASE + text)


def _alone(text, steps):
    from kh_simulations_b200.run import KHRun

    r = KHRun(_cfg(text))
    r.init()
    r.step(steps)
    s = r.state_numpy()
    r.close()
    return s


def test_batch_equals_alone(cuda):
    import torch

    from kh_simulations_b200.batch import KHBatch
    from kh_simulations_b200.run import KHRun

    steps = 7
    runs = []
    for text, _ in MIX:
        r = KHRun(_cfg(text))
        r.init()
        runs.append(r)
    b = KHBatch()
    for r in runs:
        b.add(r)
    st = torch.cuda.Stream()
    b.step(steps, st)  # 3 graph-less steps + one 4-step graph
    st.synchronize()
    b.check(st)
    for (text, _), r in zip(MIX, runs):
        assert np.array_equal(r.state_numpy(), _alone(text, steps)), text
    b.close()
    for r in runs:
        r.close()


def test_continuous_batching_membership_changes(cuda):
    """Members join and leave between batch calls; every run still ends
    bit-identical to its solo trajectory."""
    import torch

    from kh_simulations_b200.batch import KHBatch
    from kh_simulations_b200.run import KHRun

    st = torch.cuda.Stream()
    b = KHBatch()
    r0 = KHRun(_cfg(MIX[0][0]))
    r0.init()
    b.add(r0)
    b.step(5, st)
    r1 = KHRun(_cfg(MIX[1][0]))
    r1.init()
    b.add(r1)
    b.step(6, st)        # r0: 11, r1: 6
    b.remove(r0)
    r2 = KHRun(_cfg(MIX[2][0]))
    r2.init()
    b.add(r2)
    b.step(3, st)        # r1: 9, r2: 3
    st.synchronize()
    assert np.array_equal(r0.state_numpy(), _alone(MIX[0][0], 11))
    assert np.array_equal(r1.state_numpy(), _alone(MIX[1][0], 9))
    assert np.array_equal(r2.state_numpy(), _alone(MIX[2][0], 3))
    b.close()
    for r in (r0, r1, r2):
        r.close()


def test_batch_member_with_library_second_buffer(cuda):
    """A member bound with ymkh_bind_state (the library owns its second
    buffer, so an odd step count ends with a copy back to buffer 0) stays on
    its own trajectory over batch calls of odd and even length: 5 then 6
    batch steps equal 11 steps alone, for it and for a member bound with
    both buffers."""
    import ctypes as C

    import torch

    from kh_simulations_b200 import _lib
    from kh_simulations_b200.batch import KHBatch
    from kh_simulations_b200.run import KHRun

    st = torch.cuda.Stream()
    one = KHRun(_cfg(MIX[0][0]))
    one.init()
    torch.cuda.synchronize()
    b0 = one.buf[0]
    f = (C.c_void_p * 12)(*[b0[i].data_ptr() for i in range(12)])
    a = (C.c_void_p * 6)(*[b0[12 + i].data_ptr() for i in range(6)])
    bb = (C.c_void_p * 6)(*[b0[18 + i].data_ptr() for i in range(6)])
    _lib.check(one.lib.ymkh_bind_state(one.ctx, f, a, bb), "ymkh_bind_state")
    two = KHRun(_cfg(MIX[2][0]))
    two.init()
    b = KHBatch()
    b.add(one)
    b.add(two)
    b.step(5, st)
    assert one.current == 0
    b.step(6, st)
    st.synchronize()
    b.check(st)
    assert np.array_equal(one.state_numpy(), _alone(MIX[0][0], 11))
    assert np.array_equal(two.state_numpy(), _alone(MIX[2][0], 11))
    b.close()
    one.close()
    two.close()


def test_server_mix_equals_sequential(cuda):
    from kh_simulations_b200.server import KHRequest, KHServer

    reqs_a = [KHRequest(i, _cfg(t), 20 + 10 * i, arrival=0.01 * i) for i, (t, _) in enumerate(MIX[:4])]
    reqs_b = [KHRequest(i, _cfg(t), 20 + 10 * i, arrival=0.01 * i) for i, (t, _) in enumerate(MIX[:4])]
    srv = KHServer(budget_bytes=2 << 30, chunk=8, keep_state=True, check_energy=True)
    rep_b = srv.serve(reqs_a)
    rep_s = srv.serve_sequential(reqs_b)
    for a, s in zip(sorted(reqs_a, key=lambda r: r.rid), sorted(reqs_b, key=lambda r: r.rid)):
        assert a.status == s.status == "done"
        assert np.array_equal(a.state, s.state), a.rid
    assert rep_b.cell_steps == rep_s.cell_steps
    assert np.isfinite(rep_b.p50) and np.isfinite(rep_b.p99)


def test_server_large_runs_alone_equal_sequential(cuda):
    """Runs at or above large_cells are stepped alone on their own stream
    beside the batch of the smaller ones; every result still equals the
    same request run one by one, bit for bit."""
    from kh_simulations_b200.server import KHRequest, KHServer

    reqs_a = [KHRequest(i, _cfg(t), 24 + 6 * i, arrival=0.005 * i) for i, (t, _) in enumerate(MIX)]
    reqs_b = [KHRequest(i, _cfg(t), 24 + 6 * i, arrival=0.005 * i) for i, (t, _) in enumerate(MIX)]
    srv = KHServer(budget_bytes=2 << 30, chunk=8, keep_state=True, check_energy=True, large_cells=8000)
    rep = srv.serve(reqs_a)
    srv.serve_sequential(reqs_b)
    assert sum(r.cells >= 8000 for r in reqs_a) == 2
    for a, s in zip(sorted(reqs_a, key=lambda r: r.rid), sorted(reqs_b, key=lambda r: r.rid)):
        assert a.status == s.status == "done"
        assert np.array_equal(a.state, s.state), a.rid
    assert rep.extra["unfinished"] == 0


def test_server_defers_an_admission_without_room(cuda, monkeypatch):
    """A run creation that finds no device room while other runs are
    resident puts the request (and those after it) back at the head of the
    queue until runs retire; every request still completes, equal to its
    sequential run.  The lack of room is simulated on the host: the server's
    creation call reports it once."""
    from kh_simulations_b200.server import KHRequest, KHServer

    reqs_a = [KHRequest(i, _cfg(t), 16 + 4 * i, arrival=0.0) for i, (t, _) in enumerate(MIX[:4])]
    reqs_b = [KHRequest(i, _cfg(t), 16 + 4 * i, arrival=0.0) for i, (t, _) in enumerate(MIX[:4])]
    srv = KHServer(budget_bytes=2 << 30, chunk=8, keep_state=True)
    real = KHServer._start_run
    failed = []

    def flaky(self, req, stream=None, must=True):
        if not must and req.rid == 2 and not failed:
            failed.append(req.rid)
            return None  # as if creation found no room
        return real(self, req, stream, must)

    monkeypatch.setattr(KHServer, "_start_run", flaky)
    rep = srv.serve(reqs_a)
    monkeypatch.setattr(KHServer, "_start_run", real)
    srv.serve_sequential(reqs_b)
    assert failed == [2] and rep.extra["deferred_admissions"] == 1
    for a, s in zip(sorted(reqs_a, key=lambda r: r.rid), sorted(reqs_b, key=lambda r: r.rid)):
        assert a.status == s.status == "done", (a.rid, a.status)
        assert np.array_equal(a.state, s.state), a.rid


def test_autotune_runs_and_keeps_results(cuda, tmp_path, monkeypatch):
    import kh_simulations_b200.autotune as at
    from kh_simulations_b200.run import KHRun

    monkeypatch.setattr(at, "TABLE", tmp_path / "tuned.json")
    r = KHRun(_cfg(MIX[2][0]))
    r.init()
    e = at.tune(r, reps=1, graph_candidates=(2, 4))
    assert e["fct_strip"] in (32, 64, 128) and e["graph_steps"] in (2, 4)
    assert at.lookup(r.d.nx, r.d.nz, True) == e
    # tuning put the run back where it was: it continues its own trajectory
    assert r.step_count == 0
    r.step(4)
    assert np.array_equal(r.state_numpy(), _alone(MIX[2][0], 4))
    s_tuned = KHRun(_cfg(MIX[2][0]), tune=True)
    s_tuned.init()
    s_tuned.step(4)
    assert np.array_equal(s_tuned.state_numpy(), _alone(MIX[2][0], 4))
    r.close()
    s_tuned.close()


def test_runs_of_different_nz_in_one_process(cuda):
    """The column kernels' shared-memory limit is per kernel, shared by all
    runs of the process: creating a run with a smaller NZ must not lower it
    under a resident run with a larger NZ (z-mean of NZ = 2048 needs 64 KB)."""
    from kh_simulations_b200.run import KHRun

    big = KHRun(_cfg("nz_override = 2048\nnx_override = 64\nsuppress_kz0 = 1\n"))
    big.init()
    small = KHRun(_cfg("nz_override = 1600\nnx_override = 64\n"))
    small.init()
    big.step(2)
    small.step(2)
    assert np.isfinite(big.state_numpy()).all() and np.isfinite(small.state_numpy()).all()
    big.close()
    small.close()
