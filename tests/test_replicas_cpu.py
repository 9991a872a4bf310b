"""The multi-GPU form of bench.py is replicas only: every rank registers its
own copy of the workload, with no collective on the data path; the timed
region ends with a max over ranks.  Two gloo ranks on the CPU check the
sharding helper and the max-over-ranks reduction."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import bench

    dist = bench.init_group(world, "gloo")
    items = list(range(11))
    mine = bench.shard(items, rank, world)
    t = bench.reduce_max(dist, 1.5 + rank)
    out[rank] = (mine, t)
    dist.destroy_process_group()


def test_two_gloo_ranks_shard_and_max():
    world = 2
    port = _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    shards = [res[r][0] for r in range(world)]
    assert sorted(sum(shards, [])) == list(range(11))
    assert all(abs(len(a) - len(b)) <= 1 for a in shards for b in shards)
    assert all(res[r][1] == pytest.approx(1.5 + world - 1) for r in range(world))
