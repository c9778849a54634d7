"""Multi-GPU runs of bench.py are replicas: every rank holds the whole index
and answers its own query batch, and the only collective is the max of the
per-rank timings.  Exercise that host logic with two gloo ranks on the CPU,
with the oracle standing in for each rank's GPU index: each rank draws its
own batch, answers it, and the job's throughput comes from the slowest rank;
every rank's answers equal those of the same batch answered alone."""
import json
import os
import socket
import subprocess
import sys
import time

import numpy as np
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _replica(X, w, rank):
    import bench
    from falconnpp_b200 import synth
    from oracle import oracle
    Q = synth.mixture(w["nq"], w["d"], n_centres=w["n_centres"], norm_sigma=w["norm_sigma"],
                      seed=bench.query_seed(rank))
    o = oracle.Index(w["n"], w["d"])
    o.set_index_param(w["L"], w["D"], w["minSize"], w["alpha"], w["iProbes"], 1, bench.INDEX_SEED)
    o.build(X)
    o.set_qprobes(w["qprobes"])
    t0 = time.perf_counter()
    top = o.query(Q, w["k"])["topk"]
    return Q, top, (time.perf_counter() - t0) * 1000.0


def _worker(rank, world, port, q):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    from falconnpp_b200 import synth

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    w = dict(bench.WORKLOADS["mips-20Kx64-L8-tiny"], n=4000, nq=64)
    X = synth.mixture(w["n"], w["d"], n_centres=w["n_centres"], norm_sigma=w["norm_sigma"], seed=0)
    Q, top, ms = _replica(X, w, rank)
    mx = bench.reduce_max(ms, device="cpu")
    value = bench.aggregate_qps(world, w["nq"], 1, mx)
    q.put((rank, mx, value, Q.sum(), top))
    dist.barrier()
    dist.destroy_process_group()


def test_replica_host_logic_two_ranks():
    sys.path.insert(0, ROOT)
    import bench
    from falconnpp_b200 import synth
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted((q.get(timeout=180) for _ in range(2)), key=lambda r: r[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res[0][1] == res[1][1]                    # the max over ranks, on every rank
    assert res[0][2] == res[1][2] == 2 * 64 / (res[0][1] / 1000.0)
    assert not np.isclose(res[0][3], res[1][3])      # distinct query batches per replica
    # each replica's answers are those of its batch answered alone
    w = dict(bench.WORKLOADS["mips-20Kx64-L8-tiny"], n=4000, nq=64)
    X = synth.mixture(w["n"], w["d"], n_centres=w["n_centres"], norm_sigma=w["norm_sigma"], seed=0)
    for rank in range(2):
        _, alone, _ = _replica(X, w, rank)
        assert np.array_equal(alone, res[rank][4])


def test_bench_gpus_flag_spawns_replicas():
    # without torchrun, --gpus 2 starts two ranks itself; on the reference arm
    # rank 0 alone measures and prints one JSON line, rank 1 exits 0
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--workload", "mips-20Kx64-L8-tiny", "--steps", "1", "--warmup", "0"],
                       capture_output=True, text=True, timeout=600, env=env, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    j = json.loads(lines[0])
    assert j["impl"] == "reference" and j["config"]["workload"] == "mips-20Kx64-L8-tiny"
    assert j["cpu_baseline"]["kind"] in ("reference", "port")
