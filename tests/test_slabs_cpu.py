"""Host side of the z-slab decomposition (dasha_b200/slabs.py, the z-slab calls of
include/dasha_capi.h): the partition rule, the local planes of each slab and their assembly,
the NCCL id and its hand-over between ranks (2 gloo ranks), and the argument checks that need
no device."""
import ctypes as C
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from dasha_b200 import capi, slabs


def _rule(mz, n):
    rows = mz - 4
    base, extra = divmod(rows, n)
    out, first = [], 2
    for s in range(n):
        c = base + (1 if s < extra else 0)
        out.append((first, c))
        first += c
    return out


@pytest.mark.parametrize("mz,n", [(7, 1), (10, 2), (40, 2), (41, 3), (300, 8), (1028, 8), (1031, 7)])
def test_partition_covers_the_interior_rows(mz, n):
    parts = slabs.partition(mz, n)
    assert parts == _rule(mz, n)
    assert parts[0][0] == 2 and parts[-1][0] + parts[-1][1] == mz - 2
    assert all(c >= 3 for _, c in parts)
    assert max(c for _, c in parts) - min(c for _, c in parts) <= 1


@pytest.mark.parametrize("mz,n,s", [(12, 3, 0), (7, 2, 0), (40, 2, 2), (40, 2, -1), (40, 0, 0)])
def test_partition_refuses_slabs_under_three_rows(mz, n, s):
    lib = capi.load()
    f, c = C.c_int(), C.c_int()
    assert lib.dasha_slab_partition(mz, n, s, C.byref(f), C.byref(c)) == capi.E_INVALID


def test_split_and_assemble_round_trip():
    rng = np.random.default_rng(3)
    X = rng.standard_normal((8, 41, 5, 32))
    parts = slabs.partition(41, 3)
    pieces = slabs.split(X, parts)
    assert [p.shape[1] for p in pieces] == [c + 4 for _, c in parts]
    # each slab's ghost planes are its neighbours' edge rows
    assert np.array_equal(pieces[1][:, :2], pieces[0][:, -4:-2])
    assert np.array_equal(pieces[0][:, -2:], pieces[1][:, 2:4])
    assert np.array_equal(slabs.assemble(pieces, parts, 41), X)
    # the ghost planes of the pieces do not reach the assembled field
    for p in pieces:
        p[:, :2] = np.nan
        p[:, -2:] = np.nan
    pieces[0][:, :2] = X[:, :2]
    pieces[-1][:, -2:] = X[:, -2:]
    assert np.array_equal(slabs.assemble(pieces, parts, 41), X)


def test_nccl_ids_are_fresh():
    a, b = slabs.new_id(), slabs.new_id()
    assert len(a) == 128 and len(b) == 128 and a != b


def test_slab_creation_checks_need_no_device():
    from dasha_b200 import harris
    lib = capi.load()
    x, y, z = harris.make_grid(32, 8, 12, False)
    p = capi.make_params(harris.CONFIGS["c0"], 0)
    h = C.c_void_p()
    bounded = capi.GridC(32, 8, 12, capi._dp(x), capi._dp(y), capi._dp(z), (C.c_int * 3)(0, 0, 0))
    assert lib.dasha_create_slab(C.byref(bounded), C.byref(p), 2, 0, C.byref(h)) == capi.E_UNSUPPORTED
    g = capi.GridC(32, 8, 12, capi._dp(x), capi._dp(y), capi._dp(z), (C.c_int * 3)(1, 1, 0))
    assert lib.dasha_create_slab(C.byref(g), C.byref(p), 3, 0, C.byref(h)) == capi.E_INVALID   # 8 rows
    assert lib.dasha_create_slab(C.byref(g), C.byref(p), 2, 2, C.byref(h)) == capi.E_INVALID
    assert not h.value
    hs = (C.c_void_p * 2)()
    assert lib.dasha_slab_link(hs, 2) == capi.E_INVALID
    assert lib.dasha_group_stepon(hs, 1, 0.0, 1e-3, 0) == capi.E_INVALID
    assert lib.dasha_nccl_unique_id(C.create_string_buffer(64), 64) == capi.E_INVALID


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", init_method="env://", timeout=datetime.timedelta(seconds=60))
    try:
        nid = slabs.share_id(slabs.new_id, rank)
        parts = slabs.partition(1028, world)
        q.put((rank, nid, parts[rank]))
    finally:
        dist.destroy_process_group()


def test_rank_zero_id_reaches_every_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res[0][1] == res[1][1] and len(res[0][1]) == 128
    assert [r[2] for r in res] == [(2, 512), (514, 512)]


def _exchange_rank(rank, world, port, mz, q):
    """One slab per gloo rank: the global field's local planes with the ghost planes poisoned,
    then the library's exchange plan as point-to-point messages (the NCCL group's sends and
    receives, here isend/irecv of torch tensors)."""
    import datetime
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", init_method="env://", timeout=datetime.timedelta(seconds=60))
    try:
        my, mx = 3, 4
        X = np.arange(2 * mz * my * mx, dtype=np.float64).reshape(2, mz, my, mx)
        parts = slabs.partition(mz, world)
        P = slabs.split(X, parts)[rank].copy()
        first, count = parts[rank]
        if rank > 0:
            P[:, :2] = -1.0
        if rank < world - 1:
            P[:, -2:] = -1.0
        flat = [torch.from_numpy(P[f].reshape(-1)) for f in range(2)]
        reqs = []
        for f in range(2):                       # the fields in the same order on every rank
            for peer, so, ro, n in slabs.halo_plan(mz, world, rank, my * mx):
                if peer < 0:
                    continue
                reqs.append(dist.isend(flat[f][so:so + n].clone(), peer))
                buf = torch.empty(n, dtype=torch.float64)
                reqs.append((dist.irecv(buf, peer), f, ro, buf))
        for r in reqs:
            if isinstance(r, tuple):
                r[0].wait()
                flat[r[1]][r[2]:r[2] + r[3].numel()] = r[3]
            else:
                r.wait()
        got = np.stack([t.numpy().reshape(P.shape[1:]) for t in flat])
        q.put((rank, bool(np.array_equal(got, X[:, first - 2:first + count + 2]))))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,mz", [(2, 12), (3, 17)])
def test_halo_plan_exchange_between_gloo_ranks(world, mz):
    """After one exchange every slab's ghost planes hold its neighbours' edge rows: its local
    planes equal the global field's rows first-2 .. first+count+1."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_exchange_rank, args=(r, world, port, mz, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res == [(r, True) for r in range(world)]


def test_halo_plan_ranges():
    plane = 6
    for mz, n in ((12, 2), (17, 3), (1028, 8)):
        parts = slabs.partition(mz, n)
        for s, (first, count) in enumerate(parts):
            (pl, slo, rlo, c0), (pu, shi, rhi, c1) = slabs.halo_plan(mz, n, s, plane)
            assert c0 == c1 == 2 * plane
            assert pl == (s - 1 if s > 0 else -1) and pu == (s + 1 if s < n - 1 else -1)
            assert slo == 2 * plane and rlo == 0                      # own rows first, first+1 / ghosts
            assert shi == count * plane and rhi == (count + 2) * plane   # own last two rows / ghosts
