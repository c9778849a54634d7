"""The batched form (one persistent fused kernel per batch).

* FP32 precision must equal the plain path bit for bit (same hashing, same
  probes, same candidates, same canonical FP32 dot, same tie rules);
* mixed batches (per-query k and qProbes) must give every query the result
  it gets alone;
* the CUDA-graph replay must reproduce the direct launch;
* BF16 / FP8 reranking with the FP32 shortlist re-score must agree with the
  exact top-k on almost every id (recall against the plain path >= 0.97 at
  shortlist 4k) and return exact FP32 scores for the ids it returns.
"""
import numpy as np
import pytest

from falconnpp_b200 import capi, synth

pytestmark = pytest.mark.gpu


def _index(X, L, D, minSize, alpha, iProbes):
    g = capi.Index(*X.shape)
    g.set_index_param(L, D, minSize, alpha, iProbes, 8, 42)
    g.build(X)
    return g


def _batched(g, Q, k, qp, precision=0, mult=4, graph=False, ks=None, qps=None, with_val=False):
    import torch
    g.set_query_form(1, precision, mult)
    g.set_option("use_graph", int(graph))
    dq = torch.from_numpy(np.ascontiguousarray(Q)).cuda()
    kmax = int(max(ks)) if ks is not None else k
    qpmax = int(max(qps)) if qps is not None else qp
    out = torch.full((len(Q), kmax), -9, dtype=torch.int32, device="cuda")
    val = torch.zeros((len(Q), kmax), dtype=torch.float32, device="cuda")
    dk = torch.from_numpy(np.asarray(ks, np.int32)).cuda() if ks is not None else None
    dqp = torch.from_numpy(np.asarray(qps, np.int32)).cuda() if qps is not None else None
    s = torch.cuda.Stream()
    g.query_batched(dq.data_ptr(), len(Q), dk.data_ptr() if dk is not None else None,
                    dqp.data_ptr() if dqp is not None else None, kmax, qpmax, out.data_ptr(), kmax,
                    val.data_ptr(), s.cuda_stream)
    torch.cuda.synchronize()
    g.set_query_form(0, 0, 4)
    return (out.cpu().numpy(), val.cpu().numpy()) if with_val else out.cpu().numpy()


@pytest.mark.parametrize("n,d,L,D,minSize,alpha,iProbes", [
    (3000, 24, 4, 32, 20, 0.01, 1),
    (5000, 64, 6, 64, 5, 0.05, 2),
    (4000, 200, 3, 256, 50, 0.01, 3),
    (2000, 100, 5, 128, 10, 0.5, 4),
])
def test_fp32_batched_equals_plain(n, d, L, D, minSize, alpha, iProbes):
    X = synth.mixture(n, d, n_centres=16, seed=0)
    Q = synth.mixture(300, d, n_centres=16, seed=1)
    g = _index(X, L, D, minSize, alpha, iProbes)
    for qp in (1, 5, 3 * L):
        g.set_qprobes(qp)
        plain = g.query(Q, 10)
        assert np.array_equal(_batched(g, Q, 10, qp), plain), qp
        assert np.array_equal(_batched(g, Q, 10, qp, graph=True), plain), qp


def test_fp32_batched_equals_plain_with_ties():
    X = synth.p0_integer(2000, 32, xmax=7)
    Q = synth.p0_queries(60, 32, qmax=3)
    g = _index(X, 5, 32, 10, 0.02, 3)
    for qp in (2, 7, 40):
        g.set_qprobes(qp)
        assert np.array_equal(_batched(g, Q, 20, qp), g.query(Q, 20))


def test_mixed_batch_matches_alone():
    X = synth.mixture(20000, 100, n_centres=32, seed=0)
    Q = synth.mixture(400, 100, n_centres=32, seed=1)
    g = _index(X, 10, 128, 30, 0.01, 3)
    rng = np.random.default_rng(3)
    ks = rng.choice([1, 10, 100], size=len(Q))
    qps = rng.choice([5, 10, 20, 80], size=len(Q))
    for precision in (0, 1, 2):
        mixed = _batched(g, Q, 0, 0, precision=precision, ks=ks, qps=qps)
        for kk in (1, 10, 100):
            for qq in (5, 10, 20, 80):
                sel = np.where((ks == kk) & (qps == qq))[0]
                if len(sel) == 0:
                    continue
                alone = _batched(g, Q[sel], kk, qq, precision=precision)
                assert np.array_equal(mixed[sel, :kk], alone), (precision, kk, qq)
                if precision == 0:
                    g.set_qprobes(int(qq))
                    assert np.array_equal(alone, g.query(Q[sel], int(kk)))


@pytest.mark.parametrize("precision", [1, 2])
def test_low_precision_shortlist(precision):
    X = synth.mixture(50000, 200, seed=0)
    Q = synth.mixture(500, 200, seed=1)
    g = _index(X, 20, 256, 100, 0.01, 3)
    g.set_qprobes(20)
    exact = g.query(Q, 20)
    ids, val = _batched(g, Q, 20, 20, precision=precision, mult=4, with_val=True)
    rec = synth.recall_at_k(exact, ids, 20)
    assert rec >= 0.97, rec
    # returned scores are the exact FP32 scores of the returned ids
    from oracle import oracle
    mean, Xc = oracle.center(X)
    for qi in range(0, 500, 50):
        for j in range(20):
            assert val[qi, j] == np.float32(oracle.dot(Q[qi], Xc[ids[qi, j]]))


@pytest.mark.parametrize("precision", [0, 1, 2])
def test_query_order_changes_nothing(precision):
    # 3000 queries on one block per SM: the batch is a few waves, so the
    # grouped processing order is used; every query must get the result it
    # gets in submission order (and, in FP32, the plain path's)
    X = synth.mixture(20000, 200, seed=0)
    Q = synth.mixture(3000, 200, seed=1)
    g = _index(X, 10, 256, 50, 0.01, 3)
    g.set_qprobes(10)
    g.set_option("blocks_per_sm", 1)
    g.set_option("reorder_queries", 0)
    base = _batched(g, Q, 10, 10, precision=precision)
    g.set_option("reorder_queries", 1)
    for graph in (False, True):
        assert np.array_equal(_batched(g, Q, 10, 10, precision=precision, graph=graph), base), graph
    if precision == 0:
        assert np.array_equal(base, g.query(Q, 10))


@pytest.mark.parametrize("precision", [1, 2])
def test_tensor_core_rotation(precision):
    # fhtDim 256 and one probe per table (qProbes <= L / 2): the low-precision
    # modes rotate on the tensor cores with FP16 operands.  Probes may differ
    # from the exact rotation's only on near-ties, so the ids agree with the
    # exact-rotation result almost everywhere, recall against the plain path
    # stays high, and the returned scores are still exact FP32 dots.
    X = synth.mixture(50000, 200, seed=0)
    Q = synth.mixture(1000, 200, seed=1)
    g = _index(X, 40, 256, 100, 0.01, 3)
    g.set_qprobes(10)
    exact = g.query(Q, 20)
    g.set_option("tc_rotation", 0)
    ref_ids = _batched(g, Q, 20, 10, precision=precision, mult=4)
    g.set_option("tc_rotation", 1)
    ids, val = _batched(g, Q, 20, 10, precision=precision, mult=4, with_val=True)
    agree = np.mean([len(set(a) & set(b)) / 20 for a, b in zip(ref_ids.tolist(), ids.tolist())])
    assert agree >= 0.95, agree
    rec = synth.recall_at_k(exact, ids, 20)
    assert rec >= 0.95, rec
    from oracle import oracle
    mean, Xc = oracle.center(X)
    for qi in range(0, 1000, 100):
        for j in range(20):
            assert val[qi, j] == np.float32(oracle.dot(Q[qi], Xc[ids[qi, j]]))
    # the same batch again gives the same ids (the rotation is deterministic)
    assert np.array_equal(_batched(g, Q, 20, 10, precision=precision, mult=4), ids)


@pytest.mark.parametrize("precision", [0, 2])
def test_hash_set_overflow_falls_back_to_bitset(precision):
    # few, large buckets: a query's probes reach far more than the 5,120
    # unique ids the shared-memory hash set takes, so the batched kernel
    # restarts that query's gather on its L2 bitset; FP32 must still equal
    # the plain path bit for bit, and every form must be deterministic
    # (about two thirds of these queries pass the limit, so one batch runs
    # both dedupe paths)
    X = synth.mixture(40000, 64, n_centres=2, seed=0)
    Q = synth.mixture(64, 64, n_centres=2, seed=1)
    g = _index(X, 4, 64, 8000, 0.5, 2)
    g.set_qprobes(32)
    plain = g.query(Q, 10)
    st = g.stats(1)
    assert st[1] / len(Q) > 5120, st[1]  # unique candidates per query, on average past the limit
    got = _batched(g, Q, 10, 32, precision=precision, mult=4)
    if precision == 0:
        assert np.array_equal(got, plain)
    else:
        assert synth.recall_at_k(plain, got, 10) >= 0.9
    assert np.array_equal(_batched(g, Q, 10, 32, precision=precision, mult=4), got)


@pytest.mark.parametrize("precision", [0, 1, 2])
def test_host_queries_equal_device_queries(precision):
    # fpp_query with host buffers copies large batches in chunks that overlap
    # the hash kernel (whole waves of hash blocks, the last chunk the rest:
    # several chunks for these batch sizes on a B200); the results must be
    # the device-pointer path's
    import torch
    X = synth.mixture(50_000, 200, n_centres=32, seed=0)
    g = _index(X, 16, 256, 100, 0.01, 3)
    g.set_qprobes(6)
    g.set_query_form(1, precision, 2)
    for nq in (6001, 10007):
        Q = synth.mixture(nq, 200, n_centres=32, seed=1)
        for graph in (0, 1):
            g.set_option("use_graph", graph)
            host = g.query(Q, 10)
            dq = torch.from_numpy(Q).cuda()
            out = torch.zeros((len(Q), 10), dtype=torch.int32, device="cuda")
            g.query_device(dq.data_ptr(), len(Q), 10, out.data_ptr())
            torch.cuda.synchronize()
            assert np.array_equal(host, out.cpu().numpy())
            assert np.array_equal(host, g.query(Q, 10))  # the query buffer is reused safely
    g.close()
