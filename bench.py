"""Benchmark of the RK4 Hall-MHD step (the reference's stepon/setdt loop, t3dsdsc.f:136-202).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl dasha|reference]
                    [--config c0..c4] [--precision fp32|fp64] [--slabs S] [--layout replicas|slabs]

One "step" is one RK4 step (setdt + stepon) of the whole grid.  Default workload: the largest
precision-form throughput configuration, 1024x512x1024 sinh-stretched Harris sheet, FP32
perturbation state with Kahan-compensated RK4, Hall on, filter every step.  The inputs (8
fields, 17 GB in FP32) are far larger than L2, so no L2 flush is needed between steps.

`value`  cell-updates/s on the device: CUDA events on the library's stream around K steps.
`e2e`    the same metric through the C-ABI with host buffers, the reference's main loop as a
         Fortran caller runs it: dasha_set_state from host memory, K x (dasha_setdt with its
         dt read-back + dasha_stepon), dasha_get_state back to host memory.
Multi-GPU: the path does not shard (one on-device domain), so N ranks run N replicas;
`value` is the total over ranks and the time is the max over ranks.  `--layout slabs` instead
stacks the grid N times in z as one grid of N z-slabs (one per rank, ghost planes by NCCL).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "RK4 cell-updates/s"
A_STEP = {"fp32": 768.0, "fp64": 1408.0}            # algorithmic bytes per cell-update
# post-step filter, per application: read and write the state once; in FP32 the state is the
# compensated pair (x, comp), 16 values per cell
A_FILTER = {"fp32": 128.0, "fp64": 128.0}


def env_rank():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def pin_device(local_rank: int, world: int):
    """Give each rank its own GPU before the CUDA runtime of libdasha starts."""
    if world <= 1:
        return
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    devs = vis.split(",") if vis else [str(i) for i in range(64)]
    os.environ["CUDA_VISIBLE_DEVICES"] = devs[local_rank]


def max_over_ranks(value: float, dist) -> float:
    """Max of a per-rank time over all ranks (the replicas' step time is the slowest rank's)."""
    if dist is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks:
    """nvidia-smi samples during the timed region."""

    def __init__(self):
        self.p = None
        self.path = os.path.join("/tmp", f"dasha_clocks_{os.getpid()}.csv")

    def start(self):
        try:
            q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
            self.f = open(self.path, "w")
            idx = os.environ.get("CUDA_VISIBLE_DEVICES", "0").split(",")[0]
            self.p = subprocess.Popen(["nvidia-smi", "-i", idx, f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                       "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if not self.p:
            return None
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.close()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [s.strip() for s in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def build_state(cfg):
    from dasha_b200 import harris
    x, y, z = harris.make_grid(cfg.mx, cfg.my, cfg.mz, cfg.stretch)
    H = harris.gem_state_halo(x, y, z, threads=os.cpu_count() or 8)
    return x, y, z, H


def make_ctx(cfg, precision, x, y, z, H):
    from dasha_b200 import capi, harris
    d = capi.Dasha(x, y, z, capi.make_params(cfg, 0 if precision == "fp64" else 1))
    rho0, b0, p0, _ = harris.harris_profiles(z)
    d.set_equilibrium(rho0, b0, p0)
    d.set_state_halo(H)
    return d


def cpu_port_rate(steps=2, grid=(256, 128, 256), warm=0):
    """The CPU oracle (port of the reference) on the host cores: cell-updates/s."""
    from dasha_b200 import harris
    from oracle.oracle import gem_oracle
    import dataclasses
    cfg = dataclasses.replace(harris.CONFIGS["c1"], mx=grid[0], my=grid[1], mz=grid[2], filter_every=1)
    o = gem_oracle(cfg)
    t, n = 0.0, 0
    for _ in range(warm):
        dt = o.setdt()
        o.stepon(t, dt, n)
        t += dt
        n += 1
    t0 = time.perf_counter()
    for _ in range(steps):
        dt = o.setdt()
        o.stepon(t, dt, n)
        t += dt
        n += 1
    el = time.perf_counter() - t0
    return cfg.cells * steps / el, el


CPU_GRID = (256, 128, 256)     # the reduced grid of the 1024x512x1024 comparison, scaled per cell


def reference_rate(steps, warm):
    """The reference program itself (translated from its Fortran source and built in
    oracle/_ref/, its nprx x nprz MPI ranks as threads on the host cores) on the 256x128x256
    Harris/GEM grid: cell-updates/s, seconds, threads, kind and what was run.  Where no such
    build exists, the oracle restatement with OpenMP on all cores ("port")."""
    from oracle import refmodel
    cores = os.cpu_count() or 1
    mx, my, mz = CPU_GRID
    for px, pz in refmodel.BENCH_DECOMPS:
        if px * pz <= cores and os.path.exists(refmodel.ranks_path(mx, my, mz, px, pz)):
            from dasha_b200 import harris
            cfg = harris.CONFIGS["c4"]
            x, y, z = harris.make_grid(mx, my, mz, True)
            X = harris.gem_state(x, y, z)
            rho0, b0, p0, _ = harris.harris_profiles(z)
            sec, _, _ = refmodel.run_ranks(mx, my, mz, px, pz, x, y, z, X, rho0, b0, p0, cfg.eta, cfg.di, cfg.hall,
                                           cfg.cfl, warm, steps, want_state=False)
            what = (f"the reference program (t3dsdsc.f translated to C, gcc -O2) on {px}x{pz} MPI ranks as "
                    f"threads, {mx}x{my}x{mz} Harris/GEM sinh grid, its own x/y walls, {warm} warm-up + "
                    f"{steps} timed RK4 steps ({sec:.1f} s), scaled per cell")
            return mx * my * mz * steps / sec, sec, px * pz, "reference", what
    rate, el = cpu_port_rate(steps=steps, grid=CPU_GRID, warm=warm)
    what = (f"{mx}x{my}x{mz} Harris/GEM grid, {warm} warm-up + {steps} timed RK4 steps ({el:.1f} s), CPU FP64 "
            "oracle restatement with OpenMP, scaled per cell")
    return rate, el, cores, "port", what


# the reference runs at about 1 s per 1e6 cell-updates per core: each arm times a bounded
# sample of at most this many steps after at most one warm-up step
REF_MAX_STEPS = 3


def run_reference(args, rank, world):
    """The reference's CPU path on the host cores (reference_rate), each step a bounded sample:
    min(K, 3) timed steps after min(W, 1) warm-up steps on the 256x128x256 grid."""
    if rank != 0:
        return
    from dasha_b200 import harris
    steps, warm = max(1, min(args.steps, REF_MAX_STEPS)), min(args.warmup, 1)
    rate, el, cores, kind, what = reference_rate(steps, warm)
    cfg = harris.CONFIGS[args.config]
    line = {"impl": "reference", "metric": METRIC, "value": rate, "unit": "cell-updates/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * el / steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded Harris sheet + GEM perturbation)",
            "config": {"workload": cfg.name, "sample_grid": "x".join(map(str, CPU_GRID)), "precision": "fp64",
                       "timed_steps": steps, "warmup_steps": warm},
            "cpu_baseline": {"value": rate, "unit": "cell-updates/s", "cores": cores, "kind": kind, "sample": what},
            "e2e": {"value": rate, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# Profiler tags -> the __global__ instantiation they launch (several tags share one kernel:
# the current and E chains both run the 3-field radial-coefficient smoothing pass).
KERNEL_OF = {
    "k_zpv_J": "k_zpv<3 fields, radial coef, store>", "k_zpv_E": "k_zpv<3 fields, radial coef, store>",
    "k_zpv_H": "k_zpv2<3 fields, 1/8, two passes>", "k_zpv_EH": "k_zpv<6 fields, E + Hall sum>",
    "k_zpv_X": "k_zpv<4 fields, store>", "k_zpv_F": "k_zpv<4 fields, store>",
    "k_zpv_X_rk1": "k_zpv<4 fields, RK stage update>", "k_zpv_X_rk2": "k_zpv<4 fields, RK stage update>",
    "k_zpv_X_rk3": "k_zpv<4 fields, RK stage update>", "k_zpv_X_rk4": "k_zpv<4 fields, RK stage update>",
    "k_zpv_F1": "k_zpv<field pairs, compensated filter pass 1>",
    "k_zpv_F2": "k_zpv<4 fields, compensated filter pass 2>",
    "k_rhs_hydro": "k_zhydro", "k_efield_hall": "k_zeh", "k_curl": "k_zcurl<+1>",
    "k_rhs_induction": "k_zcurl<-1>", "k_cfl": "k_cfl_rate",
}


def kernel_of(tag, prec):
    """The __global__ a tag launches: the smoothing passes and the hydro RHS load their rings by
    TMA (k_zpv_tma, k_zhydro_tma) in FP64, and in FP32 for the passes of 4 and 6 fields."""
    k = KERNEL_OF.get(tag, tag)
    if k.startswith("k_zpv<") and (prec == "fp64" or not k.startswith("k_zpv<3 ")):
        return "k_zpv_tma<" + k[len("k_zpv<"):]
    if k == "k_zhydro":
        return "k_zhydro_tma"
    return k


def by_kernel(prof, prec="fp32"):
    """Group the per-tag profile {tag: (ms, launches, bytes_per_launch)} by __global__:
    {kernel: {"ms", "launches", "bytes", "tags"}} with bytes the algorithmic total."""
    out = {}
    for tag, (ms, n, b) in prof.items():
        k = kernel_of(tag, prec)
        e = out.setdefault(k, {"ms": 0.0, "launches": 0, "bytes": 0.0, "tags": []})
        e["ms"] += ms
        e["launches"] += n
        e["bytes"] += b * n
        e["tags"].append(tag)
    return out


def accuracy_c2(steps: int):
    """FP32 perturbation path against the FP64 path on the 512x256x512 sinh grid (d_i = 1,
    whistler CFL): the FP64 run takes its CFL steps, the FP32 run replays them; per field the
    relative L2 and max error of the total state, and the reconnected flux.  Then 10 timed
    steps (setdt + stepon, CUDA events) of each path for their cell-updates/s."""
    from dasha_b200 import accuracy, capi, harris
    cfg = harris.CONFIGS["c2"]
    x, y, z = harris.make_grid(cfg.mx, cfg.my, cfg.mz, cfg.stretch)
    rho0, b0, p0, _ = harris.harris_profiles(z)
    eq = np.zeros((8, cfg.mz, 1, 1))
    eq[0, :, 0, 0] = rho0
    eq[4:7, :, 0, 0] = b0
    eq[7, :, 0, 0] = p0
    H = harris.gem_state_halo(x, y, z, threads=os.cpu_count() or 8)
    ctx = {}
    for prec in (0, 1):
        d = capi.Dasha(x, y, z, capi.make_params(cfg, prec))
        d.set_equilibrium(rho0, b0, p0)
        d.set_state_halo(H)
        ctx[prec] = d
    del H
    t, dts = 0.0, []
    for n in range(steps):
        dt = ctx[0].setdt(t)
        ctx[0].stepon(t, dt, n)
        dts.append(dt)
        t += dt
    tt = 0.0
    for n, dt in enumerate(dts):
        ctx[1].stepon(tt, dt, n)
        tt += dt
    s64, s32 = ctx[0].get_state(), ctx[1].get_state()
    d64, d32 = ctx[0].diagnostics(), ctx[1].diagnostics()
    fields = accuracy.compare(s32, s64, eq)
    del s64, s32
    rate = {}
    for prec, name in ((0, "fp64"), (1, "fp32")):
        d = ctx[prec]
        tk, nk = t, steps
        for _ in range(3):
            dt = d.setdt(tk)
            d.stepon(tk, dt, nk)
            tk += dt
            nk += 1
        d.setdt(tk)
        d.timer_start()
        for _ in range(10):
            dt = d.setdt(tk)
            d.stepon(tk, dt, nk)
            tk += dt
            nk += 1
        rate[name] = cfg.cells * 10 / (d.timer_stop() / 1e3)
    for d in ctx.values():
        d.close()
    return {"workload": cfg.name, "steps": steps, "dt": "FP64 run's CFL steps replayed by the FP32 run",
            "max_rel_l2": max(v["rel_l2_total"] for v in fields.values()),
            "max_rel_max": max(v["rel_max_total"] for v in fields.values()),
            "fields": {k: {"rel_l2": v["rel_l2_total"], "rel_max": v["rel_max_total"]} for k, v in fields.items()},
            "flux_rel_err": float(abs(d32[2] - d64[2]) / abs(d64[2])),
            "cell_updates_per_s": rate, "fp32_over_fp64": rate["fp32"] / rate["fp64"]}


def run_dasha(args, rank, world):
    from dasha_b200 import harris
    dist = None
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("gloo", init_method="env://", timeout=__import__("datetime").timedelta(seconds=600))
    cfg = harris.CONFIGS[args.config]
    prec = args.precision
    x, y, z, H = build_state(cfg)
    d = make_ctx(cfg, prec, x, y, z, H)
    t, n = 0.0, 0
    for _ in range(args.warmup):
        dt = d.setdt(t)
        d.stepon(t, dt, n)
        t += dt
        n += 1
    d.setdt(t)
    if dist:
        dist.barrier()
    clocks = Clocks()
    clocks.start()
    d.timer_start()
    for _ in range(args.steps):
        dt = d.setdt(t)
        d.stepon(t, dt, n)
        t += dt
        n += 1
    ms = d.timer_stop()
    ck = clocks.stop()
    ms = max_over_ranks(ms, dist)
    cells = cfg.cells
    value = world * cells * args.steps / (ms / 1e3)

    # per-kernel breakdown: one profiled step (events around every launch)
    d.profile(True)
    dt = d.setdt(t)
    d.stepon(t, dt, n)
    prof = d.profile_read()
    d.profile(False)
    launches_per_step = sum(v[1] for v in prof.values())
    tot = sum(v[0] for v in prof.values())
    kern = by_kernel(prof, prec)
    dom_name, dom = max(kern.items(), key=lambda kv: kv[1]["ms"])
    dom_ms, dom_n = dom["ms"], dom["launches"]
    dom_bytes = dom["bytes"] / dom_n
    peak, peak_kind = peaks()
    ach = dom_bytes / (dom_ms / dom_n / 1e3) / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic_per_cell.json")
    if os.path.exists(tpath):
        try:
            tr = json.load(open(tpath))
            key = f"{dom['tags'][0]}.{prec}"
            if key in tr:
                traffic = tr[key] * cells
        except Exception:
            traffic = None
    a_step = A_STEP[prec] + A_FILTER[prec] / max(cfg.filter_every, 1)
    step_ach = a_step * (cells * args.steps / (ms / 1e3)) / 1e9

    # e2e through the C-ABI with host buffers
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    d.set_state_halo(H)
    t_set = time.perf_counter() - t0
    te, ne = 0.0, 0
    for _ in range(args.steps):
        dt = d.setdt(te)
        d.stepon(te, dt, ne)
        te += dt
        ne += 1
    d.setdt(te)   # the steps are done (the dt of the next step, read back as the loop would)
    t1 = time.perf_counter()
    from dasha_b200 import capi
    lib = d.lib
    rc = lib.dasha_get_state(d.h, H.ctypes.data_as(capi._D), H.shape[3], H.shape[2])
    if rc:
        raise capi.DashaError(rc, "get_state")
    t_get = time.perf_counter() - t1
    e2e_s = time.perf_counter() - t0
    e2e_s = max_over_ranks(e2e_s, dist)
    state_bytes = 8 * cells * 8
    e2e = {"value": world * cells * args.steps / e2e_s, "unit": "cell-updates/s",
           "h2d_bytes_per_step": state_bytes / args.steps,
           "d2h_bytes_per_step": state_bytes / args.steps + 8,
           "note": "set_state from host + K x (setdt with dt read-back + stepon) + setdt + get_state to host, wall clock",
           "set_state_s": t_set, "get_state_s": t_get,
           "set_state_GBps": state_bytes / t_set / 1e9, "get_state_GBps": state_bytes / t_get / 1e9}

    line = {"metric": METRIC, "value": value, "unit": "cell-updates/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32" if prec == "fp32" else "f64",
            "data": "synthetic (seeded Harris sheet + GEM perturbation)",
            "config": {"workload": cfg.name, "grid": [cfg.mx, cfg.my, cfg.mz], "precision": prec,
                       "state": "FP32 perturbation + Kahan RK4" if prec == "fp32" else "FP64",
                       "hall": cfg.hall, "filter_every": cfg.filter_every, "eta": cfg.eta, "di": cfg.di,
                       "dt_whistler": cfg.dt_whistler,
                       "cfl": "reference setdt + whistler speed d_i pi |B|/(rho h)" if cfg.dt_whistler
                              else "reference setdt",
                       "l2": "inputs larger than L2 (no flush)", "parallelism": f"replicas{world}"},
            "e2e": e2e,
            "gpu_launches": int(launches_per_step * args.steps),
            "roofline": {"bound": "hbm", "kernel": dom_name, "achieved": ach, "peak": peak, "unit": "GB/s",
                         "frac": ach / peak, "traffic": traffic, "peak_kind": peak_kind,
                         "bytes_per_launch": dom_bytes, "avg_launch_ms": dom_ms / dom_n,
                         "launches_per_step": dom_n, "share_of_step": dom_ms / tot},
            "step_roofline": {"algorithmic_bytes_per_cell_update": a_step, "achieved": step_ach,
                              "peak": peak, "unit": "GB/s", "frac": step_ach / peak},
            "kernels": {k: {"ms_per_step": v["ms"], "launches": v["launches"],
                            "GBps": v["bytes"] / (v["ms"] / 1e3) / 1e9,
                            "frac": v["bytes"] / (v["ms"] / 1e3) / 1e9 / peak}
                        for k, v in sorted(kern.items(), key=lambda kv: -kv[1]["ms"])},
            "tags": {k: {"ms_per_step": v[0], "launches": v[1], "GBps": v[2] * v[1] / (v[0] / 1e3) / 1e9}
                     for k, v in sorted(prof.items(), key=lambda kv: -kv[1][0])},
            "clocks": ck}
    d.close()
    del H
    if rank == 0 and world == 1 and args.acc_steps > 0 and prec == "fp32":
        # outside every timed region: the FP32 path's error against FP64, and the FP64 path's rate
        line["accuracy"] = accuracy_c2(args.acc_steps)
    if rank == 0 and world == 1 and not args.no_cpu:
        rate, el, cores, kind, what = reference_rate(REF_MAX_STEPS, 1)
        line["cpu_baseline"] = {"value": rate, "unit": "cell-updates/s", "cores": cores, "kind": kind,
                                "sample": what}
    if dist:
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_slab_group(args):
    """The grid of --config cut into --slabs z-slabs stepped as one in-process group (every slab
    on the current GPU unless several are visible): the cost of the slab machinery against the
    one-context run of the same grid.  Wall clock around K group steps, the last setdt
    synchronising every slab's stream."""
    import torch
    from dasha_b200 import harris, slabs
    cfg = harris.CONFIGS[args.config]
    ndev = max(1, torch.cuda.device_count())
    devices = [s % ndev for s in range(args.slabs)]
    grp = slabs.gem_slab_group(cfg, args.slabs, 1 if args.precision == "fp32" else 0, devices=devices)
    t, n = 0.0, 0
    for _ in range(args.warmup):
        dt = grp.setdt(t)
        grp.stepon(t, dt, n)
        t += dt
        n += 1
    dt = grp.setdt(t)
    clocks = Clocks()
    clocks.start()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        grp.stepon(t, dt, n)
        t += dt
        n += 1
        dt = grp.setdt(t)
    el = time.perf_counter() - t0
    ck = clocks.stop()
    grp.close()
    line = {"metric": METRIC, "value": cfg.cells * args.steps / el, "unit": "cell-updates/s", "n_gpus": ndev,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": el * 1e3 / args.steps,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
            "dtype": "f32" if args.precision == "fp32" else "f64",
            "data": "synthetic (seeded Harris sheet + GEM perturbation)",
            "config": {"workload": cfg.name, "grid": [cfg.mx, cfg.my, cfg.mz], "precision": args.precision,
                       "parallelism": f"zslabs{args.slabs}-in-process", "devices": devices,
                       "slab_rows": slabs.partition(cfg.mz, args.slabs),
                       "timing": "wall clock, group calls synchronise every slab"},
            "clocks": ck}
    print(json.dumps(line), flush=True)


def run_nccl_slabs(args, rank, world):
    """One z-slab per rank, one process per GPU (torchrun): the grid of --config stacked N times
    in z (N (mz-4) + 4 planes, every rank owning the one-GPU workload's mz-4 interior rows: weak
    scaling), ghost planes by NCCL inside the library.  CUDA events on each rank's stream, the
    max over ranks; value = all ranks' cell-updates / that time."""
    import datetime
    from dasha_b200 import capi, harris, slabs
    dist = None
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("gloo", init_method="env://", timeout=datetime.timedelta(seconds=600))
    cfg = harris.CONFIGS[args.config]
    mzg = world * (cfg.mz - 4) + 4
    x, y, z = harris.make_grid(cfg.mx, cfg.my, mzg, cfg.stretch)
    nid = slabs.share_id(slabs.new_id, rank) if dist else slabs.new_id()
    sl = slabs.NcclSlab(x, y, z, capi.make_params(cfg, 1 if args.precision == "fp32" else 0), rank, world, nid)
    rho0, b0, p0, _ = harris.harris_profiles(z)
    sl.set_equilibrium(rho0, b0, p0)
    first, count = sl.part
    H = harris.gem_state_halo(x, y, z, threads=os.cpu_count() or 8, planes=(first - 2, first + count + 2))
    sl.set_state_halo(H)
    del H
    t, n = 0.0, 0
    for _ in range(args.warmup):
        dt = sl.setdt(t)
        sl.stepon(t, dt, n)
        t += dt
        n += 1
    sl.setdt(t)
    if dist:
        dist.barrier()
    clocks = Clocks()
    clocks.start()
    sl.timer_start()
    for _ in range(args.steps):
        dt = sl.setdt(t)
        sl.stepon(t, dt, n)
        t += dt
        n += 1
    ms = sl.timer_stop()
    ck = clocks.stop()
    ms = max_over_ranks(ms, dist)
    sl.close()
    cells = cfg.mx * cfg.my * mzg
    line = {"metric": METRIC, "value": cells * args.steps / (ms / 1e3), "unit": "cell-updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32" if args.precision == "fp32" else "f64",
            "data": "synthetic (seeded Harris sheet + GEM perturbation)",
            "config": {"workload": f"{cfg.name} stacked x{world} in z", "grid": [cfg.mx, cfg.my, mzg],
                       "precision": args.precision, "parallelism": f"zslabs{world}-nccl",
                       "own_rows_per_rank": count, "l2": "inputs larger than L2 (no flush)"},
            "clocks": ck}
    if dist:
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="dasha", choices=["dasha", "reference"])
    ap.add_argument("--config", default="c4", choices=["c0", "c1", "c2", "c3", "c4"])
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64"])
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--acc-steps", type=int, default=100,
                    help="steps of the 512x256x512 FP32-vs-FP64 check after the timed region (0: skip)")
    ap.add_argument("--slabs", type=int, default=0,
                    help="> 1: the grid as that many z-slabs stepped as one in-process group (one process)")
    ap.add_argument("--layout", default="replicas", choices=["replicas", "slabs"],
                    help="multi-GPU form: independent replicas (default) or one z-slab per rank over NCCL")
    args = ap.parse_args()
    rank, world, local = env_rank()
    if args.slabs > 1 and args.impl == "dasha":
        run_slab_group(args)
        return
    if args.layout == "slabs" and args.impl == "dasha":
        pin_device(local, world)
        run_nccl_slabs(args, rank, world)
        return
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    pin_device(local, world)
    run_dasha(args, rank, world)


if __name__ == "__main__":
    main()
