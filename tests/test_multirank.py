"""The multi-rank host logic of bench.py, run as two gloo ranks on CPU.

bench.py under torchrun gives every rank its own stream (same generator, own
seed), no collective on the data path, and reports the whole job's throughput
from the slowest rank's time (max over ranks).  The ranks here take the same
collective steps the bench takes, with CPU tensors."""
import multiprocessing as mp
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank: int, world: int, port: int, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import datetime
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method="env://", timeout=datetime.timedelta(seconds=60))
    import bench
    from chicago_b200.synth import generate
    r, w, _ = bench.dist_env()
    step_ms = [10.0 + 5.0 * r] * 4                  # rank 1 is the slower one
    job_ms = bench.max_over_ranks(sum(step_ms), w, device="cpu")
    value = bench.job_value(w, len(step_ms), job_ms)
    first = generate(64, 48, 1, seed=bench.rank_seed(r), vmax=4.0)[0]
    q.put((r, w, job_ms, value, bench.rank_seed(r), int(first.astype(np.int64).sum())))
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_take_the_slowest_time_and_encode_their_own_streams():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    try:
        res = sorted(q.get(timeout=180) for _ in procs)
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert all(p.exitcode == 0 for p in procs)
    (r0, w0, j0, v0, s0, c0), (r1, w1, j1, v1, s1, c1) = res
    assert (r0, r1, w0, w1) == (0, 1, 2, 2)
    assert j0 == j1 == pytest.approx(60.0)           # max over ranks, seen by both
    assert v0 == v1 == pytest.approx(2 * 4 / 0.060)  # whole job: both ranks' frames over the slowest time
    assert s0 != s1 and c0 != c1                      # each rank its own seed and content
