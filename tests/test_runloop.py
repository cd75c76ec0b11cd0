"""The run loop's bookkeeping on the CPU (run.RunLoop, shared by KHRun.run
and the campaign runner), driven with a fake run whose energy is scripted:
energy checks at multiples of the energy stride, exports at step 0 and at
multiples of the export stride after the energy check of the same step,
the halt rules of ymgpu2d/main_ym.cu:467-474, and energy.csv in the
reference's format (:251-256, :458-466)."""
import math
from types import SimpleNamespace

from kh_simulations_b200.run import RunLoop


class FakeRun:
    def __init__(self, energies, dt=0.25, total=20, estride=4, xstride=10, thresh=5.0):
        self.d = SimpleNamespace(dt=dt, total_steps=total, energy_stride=estride, export_stride=xstride,
                                 energy_thresh=thresh)
        self.energies = energies  # step -> energy
        self.step_count = 0
        self.E0 = None
        self.history = []
        self.halted = False
        self.halt_reason = ""
        self.log = []

    def energy(self, stream=None):
        self.log.append(("energy", self.step_count))
        return self.energies(self.step_count)

    def mode_amp(self, k=None, stream=None):
        return (0.5 * self.step_count, 0.0)

    def step(self, n):
        assert n > 0
        self.step_count += n
        self.log.append(("step", n))

    def snapshot(self, path, fmt, stream=None):
        self.log.append(("snapshot", str(path)))

    def snapshot_wait(self):
        self.log.append(("wait",))


def drive(run, **kw):
    loop = RunLoop(run, **kw)
    try:
        loop.start()
        while not loop.finished:
            run.step(loop.steps_to_event())
            loop.after_steps()
    finally:
        loop.close()
    return loop


def test_strides_and_order(tmp_path):
    run = FakeRun(lambda s: 10.0 + s)
    seen = []
    drive(run, csv=tmp_path / "e.csv", on_export=lambda r, s: seen.append((s, len(r.history))), mode_amp=True)
    assert [r.step for r in run.history] == [0, 4, 8, 12, 16, 20]
    assert seen == [(0, 1), (10, 3), (20, 6)]  # step 20's energy check comes before its export
    steps = [n for kind, *rest in run.log if kind == "step" for n in rest]
    assert sum(steps) == 20 and steps == [4, 4, 2, 2, 4, 4]
    assert run.history[2].mode_amp == 4.0
    lines = (tmp_path / "e.csv").read_text().splitlines()
    assert lines[0] == "step,time,E_total,E_ratio"
    assert lines[1] == "0,0,1.00000000e+01,1.0"
    assert lines[2] == f"4,{4 * 0.25:.8e},{14.0:.8e},{14.0 / 10.0:.8e}"


def test_halt_on_ratio_and_nan():
    run = FakeRun(lambda s: 1.0 if s < 8 else 6.0)
    drive(run)
    assert run.halted and run.step_count == 8 and "E/E0=6.0 > 5.0" in run.halt_reason
    run = FakeRun(lambda s: 1.0 if s < 12 else math.nan)
    drive(run)
    assert run.halted and run.step_count == 12 and run.halt_reason.startswith("NaN/Inf")


def test_export_dir_writes_and_waits(tmp_path):
    run = FakeRun(lambda s: 1.0, total=25, xstride=10)
    drive(run, export_dir=tmp_path / "snaps", export_format="fp64")
    snaps = [rest[0] for kind, *rest in run.log if kind == "snapshot"]
    assert [p.rsplit("/", 1)[1] for p in snaps] == ["ym_000000.fp64", "ym_000010.fp64", "ym_000020.fp64"]
    assert run.log[-1] == ("wait",)
    assert (tmp_path / "snaps").is_dir()


def test_resume_does_not_restart_the_history():
    run = FakeRun(lambda s: 2.0, total=8)
    drive(run)
    assert len(run.history) == 3
    run.d.total_steps = 16
    drive(run)
    assert [r.step for r in run.history] == [0, 4, 8, 12, 16]
