"""The multi-GPU form of bench.py is replicas only: every rank registers its
own copy of the workload, with no collective on the data path; the timed
region ends with a barrier and a max over ranks.  Two gloo ranks on the CPU
run bench.py's process-group set-up, barrier and max-over-ranks reduction."""
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
    dist.barrier()
    t = bench.reduce_max(dist, 1.5 + rank)
    out[rank] = t
    dist.destroy_process_group()


def test_two_gloo_ranks_barrier_and_max():
    world = 2
    port = _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    assert all(res[r] == pytest.approx(1.5 + world - 1) for r in range(world))
    assert bench_single_rank_is_identity()


def bench_single_rank_is_identity():
    import bench

    return bench.init_group(1, "gloo") is None and bench.reduce_max(None, 2.5) == 2.5
