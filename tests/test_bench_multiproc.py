"""The N > 1 path of bench.py on CPU: two ranks over gloo (the GPU run uses
NCCL through the same helpers).  Ranks are independent replicas; the only
cross-rank step is the max of their timed durations."""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, out):
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench
    import torch.distributed as dist
    w, r, local = bench.dist_setup()
    assert (w, r, local) == (world, rank, rank)
    assert dist.get_backend() == "gloo"
    bench.barrier(w)
    t_ms = [30.0, 50.0][rank]                 # this rank's device time
    m = bench.reduce_max(t_ms, w)
    out.put((rank, m, bench.replica_seed(rank), bench.aggregate(1000, 10, w, m)))
    dist.destroy_process_group()


def test_two_ranks_take_the_slowest_and_sum_the_work():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, m0, s0, v0), (r1, m1, s1, v1) = got
    assert m0 == m1 == 50.0                    # max over ranks
    assert s0 != s1                            # independent replicas
    assert v0 == v1 == pytest.approx(2 * 1000 * 10 / 0.05)
