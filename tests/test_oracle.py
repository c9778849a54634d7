"""Pins the CPU oracle (the checker of every GPU parity test) against the
reference: the FWHT against the reference's own fht.c (compiled from its
sources into oracle/_ref, and the committed vectors made from it), the random
signs against the committed libstdc++ streams, and the whole index against the
committed fixtures; plus the exactness properties of the P0 fixture."""
import os

import numpy as np
import pytest

from falconnpp_b200 import synth
from oracle import oracle

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_fwht_matches_reference_vectors():
    kat = np.load(os.path.join(GOLD, "fwht_kat.npz"))
    for x, y1, y3, log_n in zip(kat["x"], kat["y1"], kat["y3"], kat["log_n"]):
        m = 1 << int(log_n)
        a = oracle.fwht(x[:m])
        assert np.array_equal(a.view(np.uint32), y1[:m].view(np.uint32))
        b = oracle.fwht(oracle.fwht(a))
        assert np.array_equal(b.view(np.uint32), y3[:m].view(np.uint32))


def test_fwht_matches_reference_build():
    ref = oracle.ref_fht()
    if ref is None:
        pytest.skip("oracle/_ref/libfht_ref.so not built (reference tree absent)")
    rng = np.random.Generator(np.random.PCG64(7))
    for log_n in range(1, 12):
        for _ in range(50):
            x = (rng.standard_normal(1 << log_n) * rng.uniform(1e-3, 1e3)).astype(np.float32)
            a = x.copy()
            ref.fht_float(a.ctypes.data, log_n)
            assert np.array_equal(a.view(np.uint32), oracle.fwht(x).view(np.uint32))


def test_rng_bits_golden():
    g = np.load(os.path.join(GOLD, "rng_bits.npz"))
    for s in g["seeds"]:
        b1, b2 = oracle.hd3_bits(int(s), 3 * 64 * 5)
        assert np.array_equal(b1, g[f"b1_{s}"]) and np.array_equal(b2, g[f"b2_{s}"])


@pytest.mark.parametrize("name", ["small_index.npz", "p0_index.npz"])
def test_index_fixture(name):
    f = np.load(os.path.join(GOLD, name))
    L, D, minSize, iProbes, qprobes, k = [int(v) for v in f["params"]]
    X, Q = f["X"], f["Q"]
    o = oracle.Index(*X.shape)
    o.set_index_param(L, D, minSize, float(f["alpha"]), iProbes, 2, 42)
    o.build(X)
    assert np.array_equal(o.center().view(np.uint32), f["center"].view(np.uint32))
    codes, scores = o.hash_codes()
    assert np.array_equal(codes, f["codes"]) and np.array_equal(scores.view(np.uint32), f["scores"].view(np.uint32))
    t = o.tables()
    assert np.array_equal(t["start"], f["start"]) and np.array_equal(t["ids"], f["ids"])
    o.set_qprobes(qprobes)
    r = o.query(Q, k, with_probes=True)
    assert np.array_equal(r["topk"], f["topk"]) and np.array_equal(r["probes"], f["probes"])


def test_p0_center_is_exactly_zero_and_dots_exact():
    X = synth.p0_integer(2048, 40, xmax=1023)
    mean, Xc = oracle.center(X)
    assert np.all(mean == 0.0) and np.array_equal(Xc, X)
    q = synth.p0_queries(1, 40, qmax=63)[0]
    exact = X.astype(np.int64) @ q.astype(np.int64)
    got = np.array([oracle.dot(q, x) for x in X[:300]])
    assert np.array_equal(got, exact[:300].astype(np.float32))


def test_bruteforce_fp64_matches_numpy():
    X = synth.mixture(3000, 24, n_centres=8, seed=5)
    Q = synth.mixture(7, 24, n_centres=8, seed=6)
    got = oracle.bf_topk_f64(X, Q, 10)
    sc = Q.astype(np.float64) @ X.astype(np.float64).T
    for i in range(len(Q)):
        order = np.lexsort((np.arange(X.shape[0]), -sc[i]))[:10]
        assert np.array_equal(got[i], order)


def test_oracle_recall_definition():
    truth = np.array([[1, 2, 3, 4], [5, 6, 7, 8]])
    ans = np.array([[4, 3, 9, 9], [5, 6, 7, 8]])
    assert synth.recall_at_k(truth, ans, 4) == pytest.approx((0.5 + 1.0) / 2)
