"""The multi-GPU path is replicas only: ranks run independent colonies and
meet once, at the end, to take the max time and the summed work.  The
aggregation is checked here with two gloo ranks on CPU."""
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


def _worker(rank, world, port, q):
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import datetime
    import torch.distributed as dist
    from baccolonygrowth_b200 import replicas
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    t, w = replicas.aggregate([1.0 + rank, 10.0 * (rank + 1)], [100.0 * (rank + 1)])
    q.put((rank, t, w, replicas.replica_seed(7, rank)))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_aggregation():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, t, w, seed in out:
        assert t == [2.0, 20.0]          # max over ranks
        assert w == [300.0]              # sum over ranks
    assert out[0][3] != out[1][3]        # independent colonies
