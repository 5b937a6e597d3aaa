"""The multi-GPU form of this path is N independent replicas (one on-device domain each, no
data-path collective); the only cross-rank step is the max of the timed region over ranks.
Exercised here with 2 gloo ranks on CPU."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", init_method="env://", timeout=datetime.timedelta(seconds=60))
    try:
        q.put((rank, bench.max_over_ranks(10.0 + 5.0 * rank, dist), bench.env_rank()))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert sorted(r[1] for r in res) == [15.0, 15.0]
    assert sorted(r[2][:2] for r in res) == [(0, 2), (1, 2)]


def test_pin_device_picks_local_rank(monkeypatch):
    import bench
    monkeypatch.setenv("CUDA_VISIBLE_DEVICES", "3,5,7")
    bench.pin_device(1, 3)
    assert os.environ["CUDA_VISIBLE_DEVICES"] == "5"
    monkeypatch.setenv("CUDA_VISIBLE_DEVICES", "2")
    bench.pin_device(0, 1)
    assert os.environ["CUDA_VISIBLE_DEVICES"] == "2"
