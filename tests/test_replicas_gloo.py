"""The N > 1 path of bench.py on the CPU: two ranks over gloo run the same
replica timing logic the GPU ranks run over NCCL (no collective on the data
path; barrier, max over ranks for the time, sum over ranks for the work)."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    import bench
    w, r, local = bench.dist_setup()
    dist.init_process_group("gloo", rank=r, world_size=w, timeout=datetime.timedelta(seconds=60))
    bench.barrier(w)
    ms = 10.0 + 5.0 * r               # each rank's own device time
    steps = 1000 * (r + 1)            # each rank's own produced steps
    t = bench.reduce_max(ms, w)       # the job takes as long as the slowest rank
    s = bench.reduce_sum(steps, w)    # whole-job work
    bench.barrier(w)
    dist.destroy_process_group()
    q.put((r, w, local, t, s, s / (t / 1e3)))


@pytest.mark.timeout(120)
def test_two_replicas_reduce_like_the_gpu_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=90) for _ in procs)
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    assert [o[:3] for o in out] == [(0, 2, 0), (1, 2, 1)]
    for _, _, _, t, s, v in out:
        assert t == 15.0 and s == 3000.0       # max of the times, sum of the work
        assert v == pytest.approx(3000 / 0.015)  # value = all ranks' units / slowest rank's time
