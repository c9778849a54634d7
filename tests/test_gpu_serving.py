"""Serving loop (continuous batching) and the batched-form autotuner.

Requests of mixed size, k and qProbes are submitted to the serving loop while
earlier ones are still running; every request must get exactly what the same
queries get alone from the batched form (and, in FP32, from the plain path),
whatever batch they were packed into, also under a tiny memory budget that
forces the admission gate to serialise them.
"""
import numpy as np
import pytest

from falconnpp_b200 import capi, synth

pytestmark = pytest.mark.gpu


def _index():
    X = synth.mixture(20000, 100, n_centres=32, seed=0)
    g = capi.Index(*X.shape)
    g.set_index_param(10, 128, 30, 0.01, 3, 8, 42)
    g.build(X)
    return g


def _alone(g, Q, k, qp, precision):
    import torch
    g.set_query_form(1, precision, 4)
    dq = torch.from_numpy(np.ascontiguousarray(Q)).cuda()
    out = torch.zeros((len(Q), k), dtype=torch.int32, device="cuda")
    g.query_batched(dq.data_ptr(), len(Q), None, None, k, qp, out.data_ptr(), k)
    return out.cpu().numpy()


@pytest.mark.parametrize("precision,budget", [(0, 1 << 30), (1, 1 << 30), (1, 4096)])
def test_server_results_match_alone(precision, budget):
    g = _index()
    Q = synth.mixture(3000, 100, n_centres=32, seed=1)
    rng = np.random.default_rng(5)
    reqs, start = [], 0
    while start < len(Q):
        n = int(rng.integers(1, 200))
        reqs.append((start, min(len(Q), start + n), int(rng.choice([1, 10, 100])), int(rng.choice([5, 10, 20, 80]))))
        start += n
    g.set_query_form(1, precision, 4)
    srv = capi.Server(g, n_streams=3, memory_budget=budget, max_batch=1024, k_max=100, qprobes_max=80)
    tickets = [srv.submit(Q[a:b], k, qp) for a, b, k, qp in reqs]
    results = [srv.wait(t) for t in tickets]
    st = srv.stats()
    srv.close()
    assert st["requests"] == len(reqs) and st["queries"] == len(Q)
    if budget < 1 << 20:
        assert st["launches"] == len(reqs)   # the gate admitted one request per batch
    else:
        assert st["launches"] < len(reqs)    # requests were packed together
    for (a, b, k, qp), (out, lat) in zip(reqs, results):
        assert lat > 0
        assert np.array_equal(out, _alone(g, Q[a:b], k, qp, precision)), (a, b, k, qp)
        if precision == 0:
            g.set_query_form(0, 0, 4)
            g.set_qprobes(qp)
            assert np.array_equal(out, g.query(Q[a:b], k))


def test_autotune_picks_an_agreeing_configuration():
    import torch
    g = _index()
    g.set_qprobes(20)
    Q = synth.mixture(2000, 100, n_centres=32, seed=2)
    dq = torch.from_numpy(Q).cuda()
    rep = g.autotune(dq.data_ptr(), len(Q), 20, 0.99)
    assert rep["tried"] >= 48 and rep["agreement"] >= 0.99 and rep["ms"] > 0
    assert rep["split_hash"] in (0, 1) and rep["reorder"] in (0, 1) and rep["precision"] in (0, 1, 2)
    out = torch.zeros((len(Q), 20), dtype=torch.int32, device="cuda")
    g.query_device(dq.data_ptr(), len(Q), 20, out.data_ptr())    # the tuned batched form
    g.set_query_form(0, 0, 4)
    exact = g.query(Q, 20)
    assert synth.recall_at_k(exact, out.cpu().numpy(), 20) >= 0.99
