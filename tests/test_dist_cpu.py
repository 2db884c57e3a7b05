"""Multi-process paths of bench.py on the CPU (gloo, world size 2): the job's
timing is the max over ranks, every rank takes the same collective steps,
and a rank that fails before a collective ends the others' wait with an
error (a short process-group timeout) instead of a hang."""
import datetime
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _init(rank, world, port, timeout_s):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=timeout_s))
    return dist


def _max_worker(rank, world, port, q):
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    dist = _init(rank, world, port, 30)
    dist.barrier()
    vals = bench.reduce_max_over_ranks([10.0 + rank, 5.0 - rank, 7.0 * (rank + 1)], dist, "cpu")
    q.put((rank, vals))
    dist.barrier()
    dist.destroy_process_group()


def _fail_worker(rank, world, port, q):
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    dist = _init(rank, world, port, 3)
    dist.barrier()
    if rank == 1:
        q.put((rank, "left"))
        q.close()
        q.join_thread()  # the message is out before the process ends
        os._exit(0)  # leaves between steps, with no collective in flight
    try:
        bench.reduce_max_over_ranks([1.0], dist, "cpu")
        q.put((rank, "returned"))
    except Exception as e:  # the wait ends with an error
        q.put((rank, "error: " + type(e).__name__))


@pytest.mark.timeout(120)
def test_max_over_ranks_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_max_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = dict(q.get(timeout=90) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert out[0] == out[1] == [11.0, 5.0, 14.0]


@pytest.mark.timeout(120)
def test_rank_failure_ends_wait_with_error():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_fail_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = dict(q.get(timeout=60) for _ in range(2))
    for p in procs:
        p.join(timeout=30)
    assert out[1] == "left"
    assert out[0].startswith("error")
