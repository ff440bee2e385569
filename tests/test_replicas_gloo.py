"""Multi-process replica logic on CPU (gloo, world size 2): unit assignment is
disjoint and covering, and the job reduction sums units and takes the
slowest rank's time -- the same helpers bench.py uses under torchrun."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from lumina_b200 import replicas


def test_assign_disjoint_covering():
    units = list(range(51))
    for world in (1, 2, 3, 8):
        parts = [replicas.assign(units, r, world) for r in range(world)]
        flat = sorted(u for p in parts for u in p)
        assert flat == units
        assert max(len(p) for p in parts) - min(len(p) for p in parts) <= 1
    with pytest.raises(ValueError):
        replicas.assign(units, 2, 2)


def test_rotated_is_permutation():
    units = [520.0, 650.0, 800.0]
    for world in (1, 2, 4):
        for r in range(world):
            assert sorted(replicas.rotated(units, r, world)) == sorted(units)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = replicas.assign(list(range(10)), rank, world)
        units, secs = replicas.reduce_job(len(mine), 1.0 + rank, dist)
        out[rank] = (mine, units, secs)
    finally:
        dist.destroy_process_group()


def test_gloo_world2_reduction():
    world = 2
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_worker, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert sorted(out[0][0] + out[1][0]) == list(range(10))
    for r in range(world):
        assert out[r][1] == 10.0 and out[r][2] == 2.0
