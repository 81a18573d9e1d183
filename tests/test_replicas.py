"""Replicas across ranks (the path does not shard: the colour-ordered spin
sweeps would need a halo exchange per colour group): bench.py's
process-group plumbing, run as two gloo ranks on the CPU.  Each rank times
its own replica; the job's time is the maximum over ranks."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    import torch.distributed as dist
    w, r, local = bench.dist_setup()
    assert (w, r, local) == (world, rank, rank)
    bench.barrier(w)
    t = bench.allmax(w, 10.0 * (rank + 1))
    q.put((rank, t))
    bench.barrier(w)
    dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_gloo_ranks_take_the_max_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(k, 2, port, q)) for k in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(90)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    got = sorted(q.get(timeout=5) for _ in range(2))
    assert got == [(0, 20.0), (1, 20.0)]


def test_single_process_needs_no_group():
    import bench
    assert bench.allmax(1, 3.5) == 3.5
    bench.barrier(1)
