"""The verified tensor-core hash of the batched form (option "tc_hash", on by default).

When every query keeps one probe per table (2 qProbes <= L, fhtDim 256,
L <= 128) the hash kernel rotates every table on the tensor cores with FP16
operands, bounds each table score's error from the query's norm, and hashes
again in the reference's FP32 arithmetic every table whose score can reach the
probe cut (src/FalconnPP.cpp:358-582); when exact scores tie at the cut it
hashes every table in FP32.  So the probes, their order and everything after
them are those of the exact hash.  Checked per query against the plain path
(pinned to the oracle by the parity tests) and against the batched form with
the option off, on mixture data of the 1M x 200 workload's shape, integer
tie-heavy data, odd and boundary table counts, n_proj below fhtDim, queries of
extreme norms and per-query qProbes; the statistics show that the FP32 re-hash
ran and covered only a share of the tables.
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


def _batched(g, Q, k, qp, precision, qps=None):
    """Batched form: ids, probes ([nq][qp_max], unordered), counts [nq][2]."""
    import torch
    g.set_query_form(1, precision, 4)
    g.set_qprobes(qp)
    dq = torch.from_numpy(np.ascontiguousarray(Q)).cuda()
    nq = len(Q)
    out = torch.full((nq, k), -9, dtype=torch.int32, device="cuda")
    s = torch.cuda.Stream()
    if qps is None:
        probes = torch.zeros((nq, qp), dtype=torch.int32, device="cuda")
        counts = torch.zeros((nq, 2), dtype=torch.int32, device="cuda")
        g.query_batched_dump(dq.data_ptr(), nq, k, out.data_ptr(), None, probes.data_ptr(), counts.data_ptr(),
                             s.cuda_stream)
        torch.cuda.synchronize()
        g.set_query_form(0, 0, 4)
        return (out.cpu().numpy(), probes.cpu().numpy().view(np.uint32).astype(np.int64),
                counts.cpu().numpy().astype(np.int64))
    dqp = torch.from_numpy(np.asarray(qps, np.int32)).cuda()
    g.query_batched(dq.data_ptr(), nq, None, dqp.data_ptr(), k, int(max(qps)), out.data_ptr(), k, None,
                    s.cuda_stream)
    torch.cuda.synchronize()
    g.set_query_form(0, 0, 4)
    return out.cpu().numpy(), None, None


def _check(g, Q, k, qp, precisions=(0, 2)):
    """tc_hash on: probes and counts equal the plain path's per query, the
    FP32 ids equal the plain path's, and every result equals tc_hash off."""
    g.set_query_form(0, 0, 4)
    g.set_qprobes(qp)
    plain = g.query_dump(Q, k, qp)
    po = np.sort(plain["probes"].astype(np.int64), axis=1)
    for prec in precisions:
        ids, probes, counts = _batched(g, Q, k, qp, prec)
        bad = np.where((np.sort(probes, axis=1) != po).any(1))[0]
        assert len(bad) == 0, f"precision {prec}, qProbes {qp}: probe sets differ for queries {bad[:5]}"
        assert np.array_equal(counts[:, 0], plain["stats"][:, 0]), (prec, qp)
        assert np.array_equal(counts[:, 1], plain["stats"][:, 1]), (prec, qp)
        if prec == 0:
            assert np.array_equal(ids, plain["topk"]), f"qProbes {qp}: FP32 top-k differs from the plain path"
        g.set_option("tc_hash", 0)
        ids0, probes0, counts0 = _batched(g, Q, k, qp, prec)
        g.set_option("tc_hash", 1)
        assert np.array_equal(ids, ids0), (prec, qp)
        assert np.array_equal(probes, probes0), (prec, qp)  # same probes in the same order
        assert np.array_equal(counts, counts0), (prec, qp)


def _rehashed(g, Q, k, qp):
    """Tables the verified hash re-hashed in FP32 (stage timing on)."""
    g.set_option("stage_timing", 1)
    _batched(g, Q, k, qp, 2)
    g.set_option("stage_timing", 0)
    return int(g.stats(1)[10])


def test_mixture_l100_equals_exact():
    # the 1M x 200 workload's shape at 200k points: L = 100, n_proj 256,
    # qProbes from 1 to 50 (2 qProbes = L) and 51 (two probes per table:
    # the exact hash)
    X = synth.mixture(200_000, 200, n_centres=256, norm_sigma=0.4, seed=0)
    Q = synth.mixture(2000, 200, n_centres=256, norm_sigma=0.4, seed=1)
    g = _index(X, 100, 256, 1000, 0.01, 3)
    for qp in (1, 2, 10, 50, 51):
        _check(g, Q, 20, qp)
    n = _rehashed(g, Q, 20, 2)
    assert 2 * len(Q) <= n < 0.5 * len(Q) * 100, n
    assert _rehashed(g, Q, 20, 51) == 0
    g.close()


def test_integer_ties_equal_exact():
    # integer sign-symmetric data: rotated coordinates and table scores tie
    # often, at the cut too (then every table is re-hashed)
    X = synth.p0_integer(4000, 200, xmax=15)
    Q = synth.p0_queries(120, 200, qmax=3)
    g = _index(X, 8, 256, 20, 0.02, 3)
    for qp in (1, 2, 3, 4):
        _check(g, Q, 20, qp)
    g.close()


@pytest.mark.parametrize("L,D", [(25, 128), (128, 256), (129, 256)])
def test_table_counts_and_nproj(L, D):
    # an odd L (the last pair of rotations repeats one table), L = 128 (the
    # largest the verified hash takes), L = 129 (exact hash), n_proj < fhtDim
    X = synth.mixture(20_000, 200, n_centres=64, seed=2)
    Q = synth.mixture(300, 200, n_centres=64, seed=3)
    g = _index(X, L, D, 50, 0.01, 3)
    for qp in (1, 5, L // 2):
        _check(g, Q, 10, qp)
    n = _rehashed(g, Q, 10, 5)
    assert (n == 0) if L > 128 else (n > 0), n
    g.close()


def test_extreme_norm_queries():
    # a zero query, norms far below and above the bound's range (every table
    # re-hashed in FP32) and just inside it (the scaled tensor-core path)
    X = synth.mixture(20_000, 200, n_centres=64, seed=4)
    base = synth.mixture(8, 200, n_centres=64, seed=5)
    scales = np.array([0.0, 1e-25, 1e-16, 1e-6, 1.0, 1e6, 1e16, 1e25], np.float32)
    Q = (base * scales[:, None]).astype(np.float32)
    g = _index(X, 16, 256, 50, 0.01, 3)
    for qp in (1, 4, 8):
        _check(g, Q, 10, qp, precisions=(0,))
    g.close()


def test_per_query_qprobes():
    # per-query qProbes within one batch: each query gets what it gets alone,
    # with the option on and off
    X = synth.mixture(50_000, 200, n_centres=128, seed=6)
    Q = synth.mixture(600, 200, n_centres=128, seed=7)
    g = _index(X, 40, 256, 100, 0.01, 3)
    rng = np.random.default_rng(8)
    qps = rng.choice([1, 2, 7, 20], size=len(Q)).astype(np.int32)
    for prec in (0, 2):
        mixed, _, _ = _batched(g, Q, 10, 20, prec, qps=qps)
        g.set_option("tc_hash", 0)
        mixed0, _, _ = _batched(g, Q, 10, 20, prec, qps=qps)
        g.set_option("tc_hash", 1)
        assert np.array_equal(mixed, mixed0), prec
        for qq in (1, 2, 7, 20):
            sel = np.where(qps == qq)[0]
            alone, _, _ = _batched(g, Q[sel], 10, int(qq), prec)
            assert np.array_equal(mixed[sel], alone), (prec, qq)
    g.close()
