"""The reference's main loop (t3dsdsc.f:97-202) over the C-ABI, with the files it writes and
when it writes them, for users without the Fortran program.

Per step: setdt (a dt below 0.1 dt0 writes m2d and stops, T:142-154), the ./data/stepnm line,
stepon (its diagn every 10 steps appends the current.dat line, T:1173-1181), nstep and time
advance, the unit-20 line (fort.20).  An output is due when time is within dt of
timein + (nst - nstin + 1) dtime and at least dnstep steps followed the last output of this
nst (T:185-199); then nst advances by nint, the restart file is written when mod(nst, 3) = 1,
and m2d and m3d always.  The loop ends after nstop steps or when nst reaches nend.  A restart
(lrstrt) reads the restart file of nst and writes m2d and m3d before the loop (T:124-129).

Beside the reference's files, `Outputs` keeps a JSON-lines run log, run.jsonl: one object per
diagn call (every 10 steps, the state after the step) with nstep, time, dt and the FP64
diagnostics of dasha_diagnostics -- mass, energy, reconnected flux, the mid-y-plane current
extrema -- and one closing object with the reason the loop ended.

    python -m dasha_b200.run --config c0 --out run_c0 --nend 3 --dtime 0.5
    python -m dasha_b200.run --config c0 --out run_c0 --nend 3 --dtime 0.5 --slabs 3   # z-slabs

On z-slabs (dasha_b200/slabs.py) the loop is the same; the whole-grid files go through host
copies of the assembled state and current.
"""
from __future__ import annotations

import argparse
import json
import os
from dataclasses import dataclass, field

from . import capi, harris, restart


@dataclass
class RunControl:
    """The reference's run-control constants (mhd03.for:1-31, t3dsdsc.f:88-93)."""
    ncase: int = 1
    nst: int = 1
    nint: int = 1
    nend: int = 5011
    dtime: float = 1.0
    dnstep: float = 10.0
    nstop: int = 900000
    lrstrt: bool = False
    write_m3d: bool = True


@dataclass
class RunResult:
    reason: str                 # "nend", "nstop" or "dt collapse"
    nstep: int
    time: float
    nst: int
    outputs: list = field(default_factory=list)   # (nstep, nst) of every output


class Outputs:
    """The files of the main loop for a GPU context, under `out_dir` as the reference lays them
    out from its working directory (restart files and current.dat, fort.20 there; m2d, m3d and
    stepnm under data/).  Method names are the reference's routines."""

    def __init__(self, d, out_dir: str):
        self.d, self.dir = d, out_dir
        self.data = os.path.join(out_dir, "data")
        os.makedirs(self.data, exist_ok=True)
        self.first_diagn = True
        self.dtlog_path = os.path.join(out_dir, "fort.20")
        if os.path.exists(self.dtlog_path):       # unit 20 starts a new file with the run
            os.remove(self.dtlog_path)
        self.runlog_path = os.path.join(out_dir, "run.jsonl")
        if os.path.exists(self.runlog_path):
            os.remove(self.runlog_path)
        self.last_diag = None

    def readin(self, nst: int):
        return restart.restore(self.d, self.dir, nst)

    def recrd(self, ncase: int, nstep: int, time: float, nst: int):
        restart.checkpoint(self.d, self.dir, ncase, nstep, time, nst)

    def recrd2(self, time: float, nst: int):
        restart.write_m2d(os.path.join(self.data, f"m2d{restart.cn(nst)}.dat"), time, self.d.x, self.d.z,
                          self.d.midplane())

    def recrd3(self, time: float, nst: int):
        restart.write_m3d_ctx(self.d, os.path.join(self.data, f"m3d{restart.cn(nst)}"), time)

    def diagn(self, time: float):
        self.last_diag = self.d.diagnostics()
        restart.write_current_dat(os.path.join(self.dir, "current.dat"), self.last_diag, time,
                                  append=not self.first_diagn)
        self.first_diagn = False

    def runlog(self, **entry):
        """One JSON line of run.jsonl; after a diagn call it carries that call's diagnostics."""
        if self.last_diag is not None and "reason" not in entry:
            names = ("mass", "energy", "flux", "jx_max", "jx_min", "jy_max", "jy_min", "jz_max", "jz_min")
            entry.update({k: float(v) for k, v in zip(names, self.last_diag)})
            self.last_diag = None
        with open(self.runlog_path, "a") as f:
            f.write(json.dumps(entry) + "\n")

    def step_begin(self, nstep: int, time: float, dt: float):
        lib = capi.load()
        restart._check(lib.dasha_stepnm_write(os.fsencode(os.path.join(self.data, "stepnm")), nstep, time, dt),
                       "stepnm write")

    def step_end(self, dt: float, time: float, nstep: int):
        lib = capi.load()
        restart._check(lib.dasha_dtlog_write(os.fsencode(self.dtlog_path), dt, time, nstep), "fort.20 write")


def main_loop(d, ctl: RunControl, out, time: float = 0.0, nstep: int = 0, log=None) -> RunResult:
    """Runs the reference's loop on context `d` with the outputs `out` (an `Outputs`)."""
    nst = ctl.nst
    res = RunResult("", nstep, time, nst)
    if ctl.lrstrt:
        _, nstep, time, nst = out.readin(nst)
        out.recrd2(time, nst)
        if ctl.write_m3d:
            out.recrd3(time, nst)
    timein, nstin = time, nst
    nstp = {}                                    # step of the last output of each nst
    while True:
        try:
            dt = d.setdt(time)
        except capi.DashaError as e:
            if e.code != capi.E_DT_COLLAPSE:
                raise                            # blow-up (the stop of diagn) or a failure
            nst += ctl.nint
            out.recrd2(time, nst)
            res.reason = "dt collapse"
            break
        if log:
            log(f"main {nstep} {time} {dt}")
        out.step_begin(nstep, time, dt)
        d.stepon(time, dt, nstep)
        if nstep % 10 == 0:
            out.diagn(time)
            if hasattr(out, "runlog"):
                out.runlog(nstep=nstep, time=time + dt, dt=dt)
        nstep += 1
        time += dt
        out.step_end(dt, time, nstep)
        if abs(time - timein - (nst - nstin + 1) * ctl.dtime) <= dt and nstep - nstp.get(nst, 0) >= ctl.dnstep:
            nstp[nst] = nstep
            nst += ctl.nint
            if nst % 3 == 1:
                out.recrd(ctl.ncase, nstep, time, nst)
            out.recrd2(time, nst)
            if ctl.write_m3d:
                out.recrd3(time, nst)
            res.outputs.append((nstep, nst))
        if nstep > ctl.nstop:
            res.reason = "nstop"
            break
        if nst >= ctl.nend:
            res.reason = "nend"
            break
    res.nstep, res.time, res.nst = nstep, time, nst
    if hasattr(out, "runlog"):
        out.runlog(reason=res.reason, nstep=nstep, time=time, nst=nst)
    return res


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--config", default="c0", choices=sorted(harris.CONFIGS))
    ap.add_argument("--precision", type=int, default=0, choices=(0, 1))
    ap.add_argument("--out", default=".")
    ap.add_argument("--nend", type=int, default=RunControl.nend)
    ap.add_argument("--dtime", type=float, default=RunControl.dtime)
    ap.add_argument("--dnstep", type=float, default=RunControl.dnstep)
    ap.add_argument("--nstop", type=int, default=RunControl.nstop)
    ap.add_argument("--restart", type=int, default=None, help="nst of the restart file to start from")
    ap.add_argument("--no-m3d", action="store_true")
    ap.add_argument("--slabs", type=int, default=0, help="> 1: the grid as that many z-slabs in this process")
    a = ap.parse_args(argv)
    ctl = RunControl(nend=a.nend, dtime=a.dtime, dnstep=a.dnstep, nstop=a.nstop, write_m3d=not a.no_m3d)
    if a.restart is not None:
        ctl.lrstrt, ctl.nst = True, a.restart
    if a.slabs > 1:
        from . import slabs
        d = slabs.gem_slab_group(harris.CONFIGS[a.config], a.slabs, a.precision)
    else:
        d = capi.gem_context(harris.CONFIGS[a.config], a.precision)
    try:
        r = main_loop(d, ctl, Outputs(d, a.out), log=print)
        print(f"{r.reason}: nstep {r.nstep}, time {r.time}, nst {r.nst}, {len(r.outputs)} outputs")
    finally:
        d.close()


if __name__ == "__main__":
    main()
