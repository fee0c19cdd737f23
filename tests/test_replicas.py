"""Host logic of multi-GPU replica runs, on two gloo ranks over CPU (no GPU).

bench.py --gpus N runs one replica per rank; its only collectives are a
barrier and the max over ranks of the timed region.  These tests run two
real ranks and check the reductions, the per-rank seeds and that a rank
which joins different inputs still reports the whole job."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from partitioned_join_b200 import replicas


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        r, w, local = replicas.world_from_env()
        ms = 10.0 + 5.0 * r                 # rank 1 is the slow one
        replicas.barrier()
        mx = replicas.max_over_ranks(ms)
        units = replicas.sum_over_ranks(1000 * (r + 1))
        rate = replicas.whole_job_rate(units, mx)
        q.put((r, w, local, replicas.replica_seed(7, r), mx, units, rate))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_reduce_timing_and_units():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(world))
    assert [x[0] for x in res] == [0, 1] and all(x[1] == 2 for x in res)
    assert res[0][3] != res[1][3]                       # replicas join different inputs
    assert all(x[4] == 15.0 for x in res)               # max over ranks
    assert all(x[5] == 3000 for x in res)               # units of the whole job
    assert all(x[6] == pytest.approx(3000 / 0.015) for x in res)


def test_single_process_is_identity():
    assert not replicas.active()
    assert replicas.max_over_ranks(3.5) == 3.5
    assert replicas.sum_over_ranks(12) == 12
    assert replicas.whole_job_rate(100, 0.0) == 0.0
