"""Multi-GPU runs of bench.py are replicas: every rank holds the whole index
and answers its own query batch, and the only collective is the max of the
per-rank timings.  Exercise that host logic with two gloo ranks on the CPU."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import datetime
    import sys

    import torch.distributed as dist
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    from falconnpp_b200 import synth

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    mx = bench.reduce_max(10.0 + rank, device="cpu")
    Qr = synth.mixture(50, 16, n_centres=4, seed=bench.query_seed(rank))
    q.put((rank, mx, Qr.sum()))
    dist.barrier()
    dist.destroy_process_group()


def test_replica_timing_reduction_two_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [11.0, 11.0]      # max over ranks on every rank
    assert not np.isclose(res[0][2], res[1][2])      # distinct query batches per replica
