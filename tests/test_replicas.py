"""Multi-GPU host logic on CPU: two gloo ranks run independent replicas and
combine only time (max) and evaluation counts (sum); results merge like the
reference's MPI gather (pyhea/model/opt.py:73-80)."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from pyhea_b200 import replicas


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ms, ev = replicas.combine(100.0 + 50.0 * rank, 1000 * (rank + 1))
        fit, occ = replicas.gather_best([0.5 - 0.1 * rank, 0.9], [[rank, 0], [rank, 1]])
        out[rank] = (ms, ev, fit, occ, replicas.replica_seed(rank, 3))
    finally:
        dist.destroy_process_group()


def test_two_rank_replicas_combine_and_merge():
    world = 2
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_rank_main, args=(world, _free_port(), out), nprocs=world, start_method="spawn", join=True)
    for rank in range(world):
        ms, ev, fit, occ, seed = out[rank]
        assert ms == 150.0 and ev == 3000.0
        assert fit == [0.4, 0.5, 0.9, 0.9]
        assert occ[0] == [1, 0] and occ[1] == [0, 0] and occ[2] == [0, 1] and occ[3] == [1, 1]
    assert out[0][4] != out[1][4]


def test_single_process_passthrough():
    assert replicas.combine(12.5, 7) == (12.5, 7.0)
    f, o = replicas.gather_best([0.3, 0.1], [[1], [2]])
    assert f == [0.1, 0.3] and o == [[2], [1]]


def test_shard_partitions_every_item_once_and_balances_work():
    work = [5, 1, 1, 1, 1, 1, 3, 2, 8, 2]
    for world in (1, 2, 3, 4, 8):
        parts = [replicas.shard(work, r, world) for r in range(world)]
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(work)))
        loads = [sum(work[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(work)
    assert replicas.shard(work, 0, 2) == replicas.shard(list(work), 0, 2)  # deterministic
    assert replicas.shard([], 0, 4) == []
