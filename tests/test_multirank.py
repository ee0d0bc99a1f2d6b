"""Host logic of the N-replica bench path, run as two gloo ranks on CPU:
process-group set-up, max-over-ranks timing and the whole-job aggregate."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    import torch
    import bench
    r, w, local = bench.dist_env()
    dist = bench.dist_init(w, use_cuda=False)
    dev = torch.device("cpu")
    bench.barrier(dist, dev)
    t_local = 0.5 + r                       # rank 1 is the slow one
    t = bench.reduce_max(dist, t_local, dev)
    value = bench.aggregate(w, 1000, 10, t)
    bench.barrier(dist, dev)
    dist.destroy_process_group()
    q.put((r, w, local, t, value))


@pytest.mark.timeout(120)
def test_two_gloo_ranks_max_timing_and_aggregate():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=90) for _ in procs)
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    for r, (rank, world, local, t, value) in enumerate(out):
        assert (rank, world, local) == (r, 2, r)
        assert t == 1.5                         # the slowest rank's time on every rank
        assert value == 2 * 1000 * 10 / 1.5     # all ranks' systems over that time


def test_single_process_needs_no_group():
    import bench
    assert bench.dist_init(1, use_cuda=False) is None
    assert bench.reduce_max(None, 3.0, None) == 3.0
    assert bench.aggregate(1, 8192, 20, 2.0) == 8192 * 20 / 2.0
