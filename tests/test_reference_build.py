"""The oracle against the reference's own code.

oracle/_ref/libfalconnpp_ref.so is the reference's src/FalconnPP.cpp,
src/Utilities.cpp and src/fht.c compiled unchanged (oracle/Makefile) against a
project-written subset of Eigen and boost::dynamic_bitset (oracle/shim/).  The
subset fixes the two reduction orders Eigen leaves to its vectoriser
(rowwise().mean() and dot()) to the documented order the oracle and the GPU
use; everything else — the sign draws, the FWHT, every priority queue, the
iLimit arithmetic and uint16 bucket sizes, the probe loop and the bitset walk
— is the reference's code.  These tests compare the oracle with it: random
signs, centred data, every bucket's ids in stored order, top-k ids, the 2D
layout (build2D / query2D), and the verbose output file.
"""
import os

import numpy as np
import pytest

from falconnpp_b200 import synth
from oracle import oracle

pytestmark = pytest.mark.skipif(oracle.ref_lib() is None, reason="reference build absent (oracle/_ref)")


def _both(X, L, D, minSize, alpha, iProbes, seed=42, threads=0):
    n, d = X.shape
    r = oracle.Reference(n, d)
    r.set_index_param(L, D, minSize, alpha, iProbes, threads, seed)
    r.build(X)
    o = oracle.Index(n, d)
    o.set_index_param(L, D, minSize, alpha, iProbes, threads, seed)
    o.build(X)
    return r, o


def _compare_index(r, o, X):
    b1r, b2r = r.bits()
    b1o, b2o = o.bits()
    assert np.array_equal(b1r, b1o) and np.array_equal(b2r, b2o), "random signs differ"
    _, Xc = oracle.center(X)
    assert np.array_equal(r.centered().view(np.uint32), Xc.view(np.uint32)), "centred data differ"
    size_r, ids_r = r.buckets()
    t = o.tables()
    assert np.array_equal(size_r, t["size"].astype(np.int64)), "bucket sizes differ"
    assert np.array_equal(ids_r, t["ids"]), "bucket contents differ"


def _compare_queries(r, o, Q, k, qps):
    for qp in qps:
        r.set_qprobes(qp)
        o.set_qprobes(qp)
        a = r.query(Q, k)
        b = o.query(Q, k)["topk"]
        bad = np.where((a != b).any(1))[0]
        assert len(bad) == 0, f"qProbes {qp}: top-k differs for queries {bad[:5]}"


def test_p0_integer_ties():
    # integer, sign-symmetric data: every order gives the same bits, ties everywhere
    X = synth.p0_integer(2000, 32, xmax=7)
    Q = synth.p0_queries(40, 32, qmax=3)
    r, o = _both(X, 5, 32, 10, 0.02, 3)
    _compare_index(r, o, X)
    assert np.all(r.centered()[0::2] == X[0::2])  # the centre is exactly 0
    _compare_queries(r, o, Q, 20, (1, 2, 7, 40))


@pytest.mark.parametrize("L,D,minSize,alpha,iProbes,qps", [
    (8, 256, 50, 0.01, 3, (10, 40, 200)),
    (6, 64, 5, 0.05, 2, (3, 30)),
    (4, 128, 20, 0.5, 4, (1, 9, 64)),
])
def test_small_mixtures(L, D, minSize, alpha, iProbes, qps):
    X = synth.mixture(12000, 100 if D != 256 else 200, n_centres=32, seed=0)
    Q = synth.mixture(150, X.shape[1], n_centres=32, seed=1)
    r, o = _both(X, L, D, minSize, alpha, iProbes)
    _compare_index(r, o, X)
    _compare_queries(r, o, Q, 10, qps)


def test_cfg1_100k():
    # the CPU-runnable configuration: 100k x 200 mixture, L=50, n_proj=256,
    # bucket_minSize=500, alpha=0.01, iProbes=1, qProbes=10, k=20
    X = synth.mixture(100_000, 200, n_centres=256, norm_sigma=0.4, seed=0)
    Q = synth.mixture(1000, 200, n_centres=256, norm_sigma=0.4, seed=1)
    r, o = _both(X, 50, 256, 500, 0.01, 1)
    _compare_index(r, o, X)
    _compare_queries(r, o, Q, 20, (10, 40))


def test_reference_2d_layout_gives_the_1d_results():
    # build2Layers / query2Layers (python build2D / query2D) store each bucket
    # as its own vector; contents and top-k equal the 1D layout's
    X = synth.mixture(8000, 64, n_centres=16, seed=0)
    Q = synth.mixture(80, 64, n_centres=16, seed=1)
    n, d = X.shape
    r1 = oracle.Reference(n, d)
    r1.set_index_param(6, 64, 10, 0.05, 2, 0, 7)
    r1.build(X)
    r2 = oracle.Reference(n, d)
    r2.set_index_param(6, 64, 10, 0.05, 2, 0, 7)
    r2.build(X, two_d=True)
    s1, i1 = r1.buckets()
    s2, i2 = r2.buckets()
    assert np.array_equal(s1, s2) and np.array_equal(i1, i2)
    for qp in (4, 20):
        r1.set_qprobes(qp)
        r2.set_qprobes(qp)
        assert np.array_equal(r1.query(Q, 10), r2.query(Q, 10))


def test_reference_verbose_file(tmp_path, capfd):
    # query(verbose=True) writes 1D_Top_<k>_D_<D>_L_<L>_iProbe_<p>_bucketMinSize_<m>
    # _bucketScale_<100 alpha>_qProbe_<q>.txt (src/FalconnPP.cpp:694-703): one
    # query per line, each id followed by a space
    X = synth.mixture(4000, 32, n_centres=8, seed=0)
    Q = synth.mixture(12, 32, n_centres=8, seed=1)
    r, o = _both(X, 4, 32, 10, 0.05, 2)
    r.set_qprobes(6)
    o.set_qprobes(6)
    cwd = os.getcwd()
    os.chdir(tmp_path)
    try:
        top = r.query(Q, 5, verbose=True)
    finally:
        os.chdir(cwd)
    out = capfd.readouterr().out
    assert "Average number of unique candidates per query" in out
    f = tmp_path / "1D_Top_5_D_32_L_4_iProbe_2_bucketMinSize_10_bucketScale_5_qProbe_6.txt"
    lines = f.read_text().split("\n")
    assert lines[-1] == "" and len(lines) == len(Q) + 1
    for q, line in enumerate(lines[:-1]):
        assert line == "".join(f"{i} " for i in top[q])
    assert np.array_equal(top, o.query(Q, 5)["topk"])
