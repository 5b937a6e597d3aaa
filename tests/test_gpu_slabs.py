"""The z-slab decomposition on a B200 (dasha_b200/slabs.py): the grid cut into 2 and 3 slabs
whose ghost planes the library refreshes between launches must reproduce the one-context run
bit for bit (every slab computes its own rows with the same operations in the same order), in
FP64 and in the FP32 compensated form, with and without the post-step filter, across the
blow-up guard's step and with the Hall term off.

All slabs of a group run on the one GPU of this test in one process (the group's host threads
order the copies against each slab's launches; no kernel waits on another).  The NCCL form is
run with one rank: its ghost exchange has no neighbour there, so this checks its loading, its
communicator and its dt reduction."""
import ctypes as C

import numpy as np
import pytest

from dasha_b200 import capi, harris, slabs

pytestmark = pytest.mark.gpu

SINH = harris.RunConfig("slab-64x12x41-sinh", 64, 12, 41, True, 0.003, 1.0, 4, dt_whistler=1)
UNIF = harris.RunConfig("slab-32x8x36", 32, 8, 36, False, 0.005, 0.5, 4)
# four slabs of the smallest size, 3 own rows each (local grids of 7 planes)
THIN = harris.RunConfig("slab-64x8x16-sinh", 64, 8, 16, True, 0.003, 1.0, 4, dt_whistler=1)


def check_diagnostics(a, b):
    """The slabs' mass, energy and flux are the one-context sums in another order (1e-12);
    the current extrema are the same values."""
    np.testing.assert_allclose(a[:3], b[:3], rtol=1e-12)
    assert np.array_equal(a[3:], b[3:]), (a[3:], b[3:])


def run(d, steps, nstep0=0):
    t, dts = 0.0, []
    for n in range(nstep0, nstep0 + steps):
        dt = d.setdt(t)
        d.stepon(t, dt, n)
        t += dt
        dts.append(dt)
    return dts, d.get_state()


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("nslabs", [2, 3])
@pytest.mark.parametrize("cfg,over", [(SINH, {}), (UNIF, {"filter_every": 3}), (UNIF, {"hall": 0})])
def test_slab_group_equals_one_context(cfg, over, nslabs, precision):
    one = capi.gem_context(cfg, precision, **over)
    grp = slabs.gem_slab_group(cfg, nslabs, precision, **over)
    try:
        assert np.array_equal(grp.get_state(), one.get_state())
        # steps 8..11: the guard (nstep % 10 == 0) runs at step 10
        d1, x1 = run(one, 4, 8)
        d2, x2 = run(grp, 4, 8)
        assert d1 == d2, (d1, d2)
        assert np.array_equal(x1, x2), np.abs(x1 - x2).max()
        assert np.array_equal(grp.current(), one.current())
        check_diagnostics(grp.diagnostics(), one.diagnostics())
    finally:
        grp.close()
        one.close()


def test_slab_calls_refused_where_they_need_the_whole_grid():
    grp = slabs.gem_slab_group(UNIF, 2, 0)
    try:
        s0 = grp.slabs[0]
        with pytest.raises(capi.DashaError) as e:
            s0.stepon(0.0, 1e-3, 0)       # a linked slab steps with its group
        assert e.value.code == capi.E_STATE
        with pytest.raises(capi.DashaError) as e:
            s0.diagnostics()              # a linked slab's diagnostics come from its group
        assert e.value.code == capi.E_STATE
        with pytest.raises(capi.DashaError) as e:
            s0.midplane()
        assert e.value.code == capi.E_UNSUPPORTED
        first, count, mzl = C.c_int(), C.c_int(), C.c_int()
        assert s0.lib.dasha_slab_rows(s0.h, C.byref(first), C.byref(count), C.byref(mzl)) == capi.OK
        assert (first.value, count.value, mzl.value) == (2, 16, 20)
        # the group still steps after the refusals
        dt = grp.setdt(0.0)
        grp.stepon(0.0, dt, 0)
    finally:
        grp.close()
    # a slab joined to nothing cannot step
    x, y, z = harris.make_grid(UNIF.mx, UNIF.my, UNIF.mz, UNIF.stretch)
    lone = slabs._Slab(capi.load(), x, y, z, capi.make_params(UNIF, 0), 2, 1, slabs.partition(UNIF.mz, 2)[1])
    try:
        rho0, b0, p0, _ = harris.harris_profiles(z)
        lone.set_equilibrium(rho0, b0, p0)
        lone.set_state(slabs.split(harris.gem_state(x, y, z), slabs.partition(UNIF.mz, 2))[1])
        with pytest.raises(capi.DashaError) as e:
            lone.setdt(0.0)
        assert e.value.code == capi.E_STATE
    finally:
        lone.close()


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("cfg,nslabs,over", [(THIN, 4, {}), (UNIF, 2, {"j0_mode": 1})], ids=["thin-4", "full-j0-2"])
def test_slab_group_edge_cases(cfg, nslabs, over, precision):
    one = capi.gem_context(cfg, precision, **over)
    grp = slabs.gem_slab_group(cfg, nslabs, precision, **over)
    try:
        d1, x1 = run(one, 6, 7)
        d2, x2 = run(grp, 6, 7)
        assert d1 == d2
        assert np.array_equal(x1, x2), np.abs(x1 - x2).max()
        check_diagnostics(grp.diagnostics(), one.diagnostics())
    finally:
        grp.close()
        one.close()


@pytest.mark.parametrize("precision", [0, 1])
def test_nccl_slab_one_rank_equals_one_context(precision):
    one = capi.gem_context(SINH, precision)
    sl = slabs.gem_nccl_slab(SINH, 0, 1, slabs.new_id(), precision)
    try:
        d1, x1 = run(one, 3, 9)
        d2, x2 = run(sl, 3, 9)
        assert d1 == d2
        assert np.array_equal(x1, x2)
        check_diagnostics(sl.diagnostics(), one.diagnostics())
    finally:
        sl.close()
        one.close()


def _nccl_rank(rank, world, port, cfg, precision, steps, q):
    import datetime
    import os
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      NCCL_NVLS_ENABLE="0")
    torch.cuda.set_device(rank)
    dist.init_process_group("gloo", init_method="env://", timeout=datetime.timedelta(seconds=120))
    try:
        nid = slabs.share_id(slabs.new_id, rank)
        sl = slabs.gem_nccl_slab(cfg, rank, world, nid, precision)
        dts, x = run(sl, steps, 8)
        q.put((rank, dts, x))
        sl.close()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("precision", [0, 1])
def test_nccl_slabs_on_several_gpus_equal_one_context(precision):
    """One process per GPU, ghost planes by NCCL (runs where at least two GPUs are visible)."""
    import socket
    import torch
    import torch.multiprocessing as mp
    world = min(torch.cuda.device_count(), 3)
    if world < 2:
        pytest.skip("needs two GPUs")
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_nccl_rank, args=(r, world, port, SINH, precision, 4, q), daemon=True)
             for r in range(world)]
    for p in procs:
        p.start()
    try:
        res = sorted((q.get(timeout=300) for _ in procs), key=lambda r: r[0])
        for p in procs:
            p.join(timeout=120)
            assert p.exitcode == 0
    finally:
        for p in procs:   # a rank still waiting in a collective does not outlive the test
            if p.is_alive():
                p.kill()
                p.join(timeout=30)
    one = capi.gem_context(SINH, precision)
    try:
        d1, x1 = run(one, 4, 8)
    finally:
        one.close()
    parts = slabs.partition(SINH.mz, world)
    assert all(r[1] == d1 for r in res)
    assert np.array_equal(slabs.assemble([r[2] for r in res], parts, SINH.mz), x1)


def test_main_loop_on_slabs_writes_the_files_of_one_context(tmp_path):
    """The reference's main loop (dasha_b200/run.py) on 3 slabs writes the files of the
    one-context run byte for byte: restart files, m2d, m3d, current.dat, stepnm, fort.20 (a
    group's outputs go through host copies of the assembled state; the one context streams
    them and also writes its exact-resume records, *.state, which a group does not)."""
    import json
    import os
    from dasha_b200 import run
    one = capi.gem_context(UNIF, 0)
    grp = slabs.gem_slab_group(UNIF, 3, 0)
    try:
        dt0 = capi.gem_context(UNIF, 0).setdt(0.0)
        res = []
        for d, name in ((one, "one"), (grp, "slabs")):
            ctl = run.RunControl(nend=5, dtime=4 * dt0, dnstep=2)
            res.append(run.main_loop(d, ctl, run.Outputs(d, str(tmp_path / name))))
        a, b = res
        assert (a.reason, a.nstep, a.time, a.nst, a.outputs) == (b.reason, b.nstep, b.time, b.nst, b.outputs)

        def files(root):
            out = []
            for dp, _, fs in os.walk(root):
                out += [os.path.relpath(os.path.join(dp, f), root) for f in fs
                        if not f.endswith(".state") and f != "run.jsonl"]
            return sorted(out)

        fa, fb = files(tmp_path / "one"), files(tmp_path / "slabs")
        assert fa == fb and len(fa) >= 6, (fa, fb)
        assert any(f.startswith("mhd") for f in fa)
        for f in fa:
            assert (tmp_path / "one" / f).read_bytes() == (tmp_path / "slabs" / f).read_bytes(), f
        ja = [json.loads(x) for x in open(tmp_path / "one" / "run.jsonl")]
        jb = [json.loads(x) for x in open(tmp_path / "slabs" / "run.jsonl")]
        assert len(ja) == len(jb)
        for x, y in zip(ja, jb):
            assert x.keys() == y.keys()
            for k in x:
                if k in ("mass", "energy", "flux"):
                    assert abs(x[k] - y[k]) <= 1e-12 * abs(x[k]), (k, x[k], y[k])
                else:
                    assert x[k] == y[k], (k, x[k], y[k])
    finally:
        grp.close()
        one.close()
