"""bench.py at N > 1 runs replicas: every rank processes its own seeded batch
and the job's rate is world x points over the slowest rank's step time.  Two
`gloo` ranks on the CPU check the rank-side pieces: the all-reduce MAX of the
step time and the whole-job rate (bench.replica_rate), and that each rank draws
a different batch of the same workload (workloads.bench_seed)."""
import os
import socket

import numpy as np

import bench
from vecgeom_b200 import workloads as W


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, q) -> None:
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        # rank r takes (r + 1) ms per step over 1,000,000 point-ops
        step_ms, value = bench.replica_rate(1_000_000, float(rank + 1), world, dist, device="cpu")
        spec = W.config2_shapes()["tube"]
        wl = W.make_workload(spec, 256, W.bench_seed(0, rank))
        q.put((rank, step_ms, value, wl.x.tolist()))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_reduce_the_step_time_and_draw_their_own_batches():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = {}
    for _ in procs:
        r, step_ms, value, xs = q.get(timeout=120)
        got[r] = (step_ms, value, np.array(xs))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in (0, 1):
        step_ms, value, _ = got[r]
        assert step_ms == 2.0                      # the slower rank's step
        assert abs(value - 2 * 1_000_000 / 2e-3 / 1e6) < 1e-9   # 1,000 Mpoint-ops/s
    assert not np.array_equal(got[0][2], got[1][2])  # each rank its own batch
    # one rank alone: its own step time and points
    assert bench.replica_rate(1_000_000, 2.0, 1) == (2.0, 500.0)
