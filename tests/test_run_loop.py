"""The reference's main loop (dasha_b200/run.py, t3dsdsc.f:97-202) on the host, with a fake
context: the output cadence, the restart-file rule mod(nst, 3) = 1, the diagn lines every 10
steps, the dt-collapse stop and the restart entry, against step numbers worked out by hand
from the reference's conditions; and the file names and contents that `Outputs` writes."""
import ctypes
import os

import numpy as np
import pytest

from dasha_b200 import capi, run
from oracle import fortran_io as fio


class FakeContext:
    """setdt gives `dt` (or raises E_DT_COLLAPSE from call `collapse_at` on); stepon records."""

    def __init__(self, dt=0.25, collapse_at=None, mx=8, mz=6):
        self.dt, self.collapse_at, self.calls, self.steps = dt, collapse_at, 0, []
        self.x, self.z = np.linspace(0, 1, mx), np.linspace(-1, 1, mz)
        self.mx, self.mz = mx, mz

    def setdt(self, time):
        self.calls += 1
        if self.collapse_at is not None and self.calls >= self.collapse_at:
            raise capi.DashaError(capi.E_DT_COLLAPSE, "dt fell below 0.1*dt0")
        return self.dt

    def stepon(self, time, dt, nstep):
        self.steps.append((nstep, time, dt))

    def diagnostics(self):
        return np.arange(capi.NDIAG, dtype=float) + 1.0

    def midplane(self):
        return np.ones((11, self.mz, self.mx))


class Recorder:
    def __init__(self):
        self.log = []

    def __getattr__(self, name):
        def rec(*a, **kw):
            self.log.append((name,) + a + ((kw,) if kw else ()))
            return (1, 40, 10.0, 5) if name == "readin" else None
        return rec

    def names(self, name):
        return [e[1:] for e in self.log if e[0] == name]


def test_output_cadence():
    d, out = FakeContext(dt=0.25), Recorder()
    r = run.main_loop(d, run.RunControl(nend=6, dtime=1.0, dnstep=3), out)
    # |0.25 n - k| <= 0.25 with n - nstp(nst) >= 3: the first n of each window k = 1..5
    assert r.outputs == [(3, 2), (7, 3), (11, 4), (15, 5), (19, 6)]
    assert (r.reason, r.nstep, r.time, r.nst) == ("nend", 19, 4.75, 6)
    assert out.names("recrd") == [(1, 11, 2.75, 4)]                     # mod(nst, 3) = 1
    assert [a[1] for a in out.names("recrd2")] == [2, 3, 4, 5, 6]
    assert [a[1] for a in out.names("recrd3")] == [2, 3, 4, 5, 6]
    assert out.names("diagn") == [(0.0,), (2.5,)]                        # nstep 0 and 10, pre-step time
    assert out.names("step_begin")[:2] == [(0, 0.0, 0.25), (1, 0.25, 0.25)]
    assert out.names("step_end")[-1] == (0.25, 4.75, 19)
    assert [s[0] for s in d.steps] == list(range(19))


def test_dnstep_holds_back_an_early_window():
    # dt = 0.5, dtime = 1: the window k = 1 opens at n = 1 (|0.5 - 1| <= 0.5) but dnstep = 2
    # waits for n = 2; then k = 2 opens at n = 3, and n - nstp(2) = 3 >= 2
    r = run.main_loop(FakeContext(dt=0.5), run.RunControl(nend=3, dtime=1.0, dnstep=2), Recorder())
    assert r.outputs == [(2, 2), (3, 3)]


def test_nstop_and_dt_collapse():
    r = run.main_loop(FakeContext(dt=0.25), run.RunControl(nend=100, dtime=1.0, dnstep=3, nstop=5), Recorder())
    assert (r.reason, r.nstep) == ("nstop", 6)
    out = Recorder()
    r = run.main_loop(FakeContext(dt=0.25, collapse_at=5), run.RunControl(nend=100, dtime=1.0, dnstep=3), out)
    assert (r.reason, r.nstep, r.nst) == ("dt collapse", 4, 3)           # one output at n = 3, then nst + 1
    assert [a[1] for a in out.names("recrd2")] == [2, 3]
    with pytest.raises(capi.DashaError):                                 # a blow-up stops the loop
        class Blow(FakeContext):
            def setdt(self, time):
                raise capi.DashaError(capi.E_BLOWUP, "max Jy")
        run.main_loop(Blow(), run.RunControl(), Recorder())


def test_restart_entry():
    out = Recorder()
    r = run.main_loop(FakeContext(dt=0.25), run.RunControl(nst=5, lrstrt=True, nend=6, dtime=1.0, dnstep=3), out)
    assert out.log[0] == ("readin", 5)
    assert out.log[1][:3] == ("recrd2", 10.0, 5) and out.log[2][:3] == ("recrd3", 10.0, 5)
    # timein = 10, nstin = 5, nstep from the file (40): the window k = 1 opens at time 10.75
    assert r.outputs == [(43, 6)] and r.reason == "nend"


class FakeLib:
    """The C-ABI calls that the context-bound writers make, recorded."""

    def __init__(self):
        self.calls = []

    def dasha_checkpoint(self, h, path, ncase, nstep, time, nst, maxsub):
        self.calls.append(("checkpoint", os.fsdecode(path), ncase, nstep, time, nst))
        return 0

    def dasha_m3d_write_ctx(self, h, path, time):
        self.calls.append(("m3d", os.fsdecode(path), time))
        return 0

    def dasha_restore(self, h, path, ncase, nstep, time, nst):
        self.calls.append(("restore", os.fsdecode(path)))
        for ref, v in ((ncase, 1), (nstep, 40), (time, 10.0), (nst, 5)):
            ref._obj.value = v
        return 0


class FakeBound(FakeContext):
    def __init__(self):
        super().__init__()
        self.lib, self.h = FakeLib(), None
        self.states = []

    def _check(self, rc):
        assert rc == 0

    def set_state(self, X):
        self.states.append(X.shape)


def test_outputs_files(tmp_path):
    d = FakeBound()
    out = run.Outputs(d, str(tmp_path))
    r = run.main_loop(d, run.RunControl(nend=5, dtime=1.0, dnstep=3), out)
    assert r.outputs == [(3, 2), (7, 3), (11, 4), (15, 5)]
    data = tmp_path / "data"
    assert sorted(os.listdir(data)) == ["m2d002.dat", "m2d003.dat", "m2d004.dat", "m2d005.dat", "stepnm"]
    assert ("checkpoint", os.path.join(str(tmp_path), "mhd004000"), 1, 11, 2.75, 4) in d.lib.calls
    assert ("m3d", os.path.join(str(data), "m3d005"), 3.75) in d.lib.calls
    # current.dat: nstep 0 and 10; stepnm and fort.20: one line per step
    diag = d.diagnostics()
    assert (tmp_path / "current.dat").read_text() == (fio.current_dat_line(*diag[3:9], 0.0)
                                                      + fio.current_dat_line(*diag[3:9], 2.5))
    assert (data / "stepnm").read_text() == "".join(fio.stepnm_line(n, 0.25 * n, 0.25) for n in range(15))
    assert (tmp_path / "fort.20").read_text() == "".join(fio.dtlog_line(0.25, 0.25 * n, n) for n in range(1, 16))
    m2d = (data / "m2d003.dat").read_text()
    assert m2d == fio.m2d_text(1.75, d.x, d.z, np.ones((8, d.mz, 1, d.mx)), np.ones((3, d.mz, 1, d.mx)))
    # run.jsonl: the diagnostics after steps 0 and 10 (the diagn steps), then the end of the run
    import json
    log = [json.loads(line) for line in (tmp_path / "run.jsonl").read_text().splitlines()]
    assert [e.get("nstep") for e in log] == [0, 10, 15]
    assert log[0]["time"] == 0.25 and log[0]["dt"] == 0.25 and log[1]["time"] == 2.75
    for e in log[:2]:
        assert [e[k] for k in ("mass", "energy", "flux", "jx_max", "jx_min", "jy_max", "jy_min", "jz_max",
                               "jz_min")] == list(diag)
    assert log[2] == {"reason": "nend", "nstep": 15, "time": 3.75, "nst": 5}
    # a second run in the same directory starts fort.20 and current.dat over, appends stepnm
    d2 = FakeBound()
    run.main_loop(d2, run.RunControl(nend=2, dtime=1.0, dnstep=3), run.Outputs(d2, str(tmp_path)))
    assert len((tmp_path / "fort.20").read_text().splitlines()) == 3
    assert len((tmp_path / "current.dat").read_text().splitlines()) == 1
    assert len((data / "stepnm").read_text().splitlines()) == 15 + 3
    # the restart entry reads mhdNNN000 through dasha_restore
    d3 = FakeBound()
    run.main_loop(d3, run.RunControl(nst=5, lrstrt=True, nend=6, dtime=1.0, dnstep=3), run.Outputs(d3, str(tmp_path)))
    assert d3.lib.calls[0] == ("restore", os.path.join(str(tmp_path), "mhd005000"))
