"""Multi-process (world size 2, gloo, CPU) checks of the benchmark's N > 1
logic: replicas get distinct frame streams, the timing reduction is a max over
ranks, and the whole-job ms/frame divides the slowest rank's time by all
frames processed.  No GPU is used: the path has no data-path collective, so
this is all the multi-rank logic there is."""
import os
import socket

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world)
    r, w, local = bench.rank_env()
    local_ms = 10.0 * (rank + 1)  # rank 1 is the slower replica
    m = bench.max_over_ranks(local_ms, dist)
    seeds = [None] * world
    dist.all_gather_object(seeds, bench.frame_seed(r))
    q.put((rank, r, w, local, m, seeds, bench.whole_job_ms_per_frame(m, 5, w)))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_reduction_and_partition():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    results = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, r, w, local, m, seeds, job in results:
        assert (r, w, local) == (rank, 2, rank)
        assert m == 20.0                     # max over ranks
        assert len(set(seeds)) == 2          # each replica has its own frames
        assert job == 20.0 / (5 * 2)
