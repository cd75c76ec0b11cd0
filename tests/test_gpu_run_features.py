"""Run-level features around the step: exact checkpoints, the halt rule on
a host-injected NaN, the mode-amplitude record of the run loop, and
withdrawing a served request mid-flight.  Faults are made on the host
(a prepared state, a request's cancel time); nothing faults the GPU."""
import math

import numpy as np
import pytest

from cases import BASE

pytestmark = pytest.mark.gpu

SMALL = BASE + "nz_override = 64\nnx_override = 128\nkz_keep_max = 21\n"


def _run(text=SMALL):
    from kh_simulations_b200.config import loads
    from kh_simulations_b200.run import KHRun

    return KHRun(loads(text))


def test_checkpoint_resume_is_exact(cuda, tmp_path):
    a = _run()
    a.init()
    a.run(total_steps=7, energy_stride=5, mode_amp=True)
    a.save_checkpoint(tmp_path / "ck.npz")
    b = _run()
    b.load_checkpoint(tmp_path / "ck.npz")
    assert b.step_count == 7 and b.E0 == a.E0 and len(b.history) == len(a.history)
    a.run(total_steps=20, energy_stride=5, mode_amp=True)
    b.run(total_steps=20, energy_stride=5, mode_amp=True)
    assert np.array_equal(a.state_numpy(), b.state_numpy())
    assert [(r.step, r.energy, r.mode_amp) for r in a.history] == [(r.step, r.energy, r.mode_amp) for r in b.history]
    a.close()
    b.close()


def test_checkpoint_rejects_other_grid(cuda, tmp_path):
    a = _run()
    a.init()
    a.save_checkpoint(tmp_path / "ck.npz")
    b = _run(BASE + "nz_override = 32\nnx_override = 128\n")
    with pytest.raises(ValueError, match="grid"):
        b.load_checkpoint(tmp_path / "ck.npz")
    a.close()
    b.close()


def test_host_injected_nan_halts_the_run(cuda):
    """A NaN planted in a host-prepared initial state: the run stops at the
    first energy check with the reference's NaN/Inf halt."""
    r = _run()
    r.init()
    st = r.state_numpy()
    st[13, 10, 20] = np.nan  # px of beam A
    r.set_state(st)
    r.E0 = None
    hist = r.run(total_steps=50, energy_stride=10)
    assert r.halted and "NaN" in r.halt_reason
    assert hist[-1].step == 10 and r.step_count == 10


def test_mode_amp_recorded_at_the_energy_stride(cuda):
    r = _run()
    r.init()
    hist = r.run(total_steps=20, energy_stride=10, mode_amp=True)
    assert [h.step for h in hist] == [0, 10, 20]
    assert all(math.isfinite(h.mode_amp) and h.mode_amp > 0 for h in hist)
    assert hist[-1].mode_amp == r.mode_amp()[0]
    r.close()


def test_served_request_withdrawn_mid_flight(cuda):
    """A request withdrawn after admission is retired between chunks with
    status 'cancelled' (its memory freed); the others complete with the same
    results as when served one by one."""
    from kh_simulations_b200.config import loads
    from kh_simulations_b200.server import KHRequest, KHServer

    ticks = iter(float(i) for i in range(10 ** 6))

    def clock():  # deterministic: every call advances one second
        return next(ticks)

    def reqs():
        return [KHRequest(0, loads(SMALL), 60, 0.0), KHRequest(1, loads(SMALL.replace("64", "32", 1)), 60, 0.0),
                KHRequest(2, loads(SMALL), 60, 0.0, cancel_at=4.0)]

    srv = KHServer(1 << 30, chunk=10, clock=clock)
    served = srv.serve(reqs())
    st = {r.rid: r.status for r in served.requests}
    assert st == {0: "done", 1: "done", 2: "cancelled"}
    assert served.summary()["cancelled"] == 1
    seq = KHServer(1 << 30, chunk=10).serve_sequential([r for r in reqs() if r.rid != 2])
    e_seq = {r.rid: r.energy for r in seq.requests}
    for r in served.requests:
        if r.status == "done":
            assert r.energy == e_seq[r.rid]
