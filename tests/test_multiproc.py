"""World-size-2 gloo test (CPU) of the replica path of bench.py: every rank
times its own independent merge, the job's step time is the maximum over
ranks and its throughput counts all ranks' work."""
import os
import socket
import sys
from pathlib import Path

import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    ms = 10.0 + 5.0 * rank  # rank 1 is the slow one
    worst = bench.max_over_ranks(ms, world)
    value = bench.job_throughput(1 << 27, world, worst)
    bench.barrier(world)
    q.put((rank, worst, value))
    dist.destroy_process_group()


def test_replicas_max_over_ranks_gloo():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, worst, value in out:
        assert worst == 15.0
        assert abs(value - 2 * (1 << 27) / 0.015) < 1.0
