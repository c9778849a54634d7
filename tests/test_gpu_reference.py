"""The CUDA path against the reference's own code (not only the oracle).

oracle/_ref/libfalconnpp_ref.so is the reference's src/FalconnPP.cpp and
src/Utilities.cpp compiled unchanged (with the Eigen / Boost subset of
oracle/shim/, whose mean and dot follow the documented order the GPU uses).
Here the GPU index and queries are compared with it directly:

* through the C ABI: every bucket's ids in stored order, and top-k ids;
* through the pybind module with the reference's class API: build / query
  against build2Layers_1D / query2Layers_1D, and build2D / query2D against
  the reference's 2D layout (build2Layers / query2Layers), which give the
  same results;
* query(verbose=True): the statistics lines and the 1D_Top_...txt file
  (src/FalconnPP.cpp:682-703) equal the reference's, byte for byte.
"""
import os

import numpy as np
import pytest

from falconnpp_b200 import capi, synth
from oracle import oracle

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(oracle.ref_lib() is None, reason="reference build absent (oracle/_ref)")]


def _reference(X, L, D, minSize, alpha, iProbes, seed=42, threads=0, two_d=False):
    r = oracle.Reference(*X.shape)
    r.set_index_param(L, D, minSize, alpha, iProbes, threads, seed)
    r.build(X, two_d=two_d)
    return r


def _gpu_buckets(g):
    start, ids = g.dump_tables()
    return np.diff(start.astype(np.int64)), ids


@pytest.mark.parametrize("case", ["p0", "mixture", "cfg1"])
def test_capi_equals_reference(case):
    if case == "p0":
        X, Q = synth.p0_integer(2000, 32, xmax=7), synth.p0_queries(40, 32, qmax=3)
        prm, qps, k = (5, 32, 10, 0.02, 3), (2, 7, 40), 20
    elif case == "mixture":
        X, Q = synth.mixture(12000, 200, n_centres=32, seed=0), synth.mixture(200, 200, n_centres=32, seed=1)
        prm, qps, k = (8, 256, 50, 0.01, 3), (10, 40, 200), 10
    else:
        X = synth.mixture(100_000, 200, n_centres=256, norm_sigma=0.4, seed=0)
        Q = synth.mixture(1000, 200, n_centres=256, norm_sigma=0.4, seed=1)
        prm, qps, k = (50, 256, 500, 0.01, 1), (10,), 20
    r = _reference(X, *prm)
    g = capi.Index(*X.shape)
    g.set_index_param(*prm, 8, 42)
    g.build(X)
    size_r, ids_r = r.buckets()
    size_g, ids_g = _gpu_buckets(g)
    assert np.array_equal(size_r, size_g), "bucket sizes differ from the reference"
    assert np.array_equal(ids_r, ids_g), "bucket contents differ from the reference"
    for qp in qps:
        r.set_qprobes(qp)
        g.set_qprobes(qp)
        ref = r.query(Q, k)
        got = g.query(Q, k)
        bad = np.where((ref != got).any(1))[0]
        assert len(bad) == 0, f"qProbes {qp}: top-k differs from the reference for queries {bad[:5]}"
    g.close()


def test_pybind_class_and_2d_aliases_equal_reference():
    from falconnpp_b200 import FalconnPP
    X = synth.mixture(10000, 64, n_centres=16, seed=0)
    Q = synth.mixture(100, 64, n_centres=16, seed=1)
    n, d = X.shape
    prm = dict(n_tables=6, n_proj=64, bucket_minSize=10, bucket_scale=0.05, iProbes=2)
    r1 = _reference(X, 6, 64, 10, 0.05, 2, seed=7)
    r2 = _reference(X, 6, 64, 10, 0.05, 2, seed=7, two_d=True)
    idx = FalconnPP.FalconnPP(n, d)
    idx.setIndexParam(**prm, random_seed=7)
    idx.build(np.transpose(X))  # (d, n): the reference's column-major layout, no copy
    idx2 = FalconnPP.FalconnPP(n, d)
    idx2.setIndexParam(**prm, n_threads=4, random_seed=7)
    idx2.build2D(np.transpose(X))
    for qp in (4, 20):
        r1.set_qprobes(qp)
        r2.set_qprobes(qp)
        idx.set_qProbes(qp)
        idx2.set_qProbes(qp)
        a = idx.query(np.transpose(Q), 10)
        b = idx2.query2D(np.transpose(Q), n_neighbors=10)
        assert a.dtype == np.int32 and a.shape == (len(Q), 10)
        assert np.array_equal(a, r1.query(Q, 10)), qp
        assert np.array_equal(b, r2.query(Q, 10)), qp
    idx.clear()
    with pytest.raises(RuntimeError):
        idx.query(np.transpose(Q), 10)


def _stat_lines(text):
    return [l for l in text.splitlines() if l.startswith("Average number of")]


def test_verbose_output_equals_reference(tmp_path, capfd):
    from falconnpp_b200 import FalconnPP
    X = synth.mixture(6000, 48, n_centres=8, seed=0)
    Q = synth.mixture(50, 48, n_centres=8, seed=1)
    n, d = X.shape
    # one host thread: the reference counts empty buckets outside its
    # OpenMP reduction, so only a single-threaded run gives exact counts
    r = _reference(X, 4, 64, 10, 0.05, 2, seed=5, threads=1)
    r.set_qprobes(12)
    idx = FalconnPP.FalconnPP(n, d)
    idx.setIndexParam(4, 64, 10, 0.05, 2, random_seed=5)
    idx.build(np.transpose(X))
    idx.set_qProbes(12)
    fname = "1D_Top_7_D_64_L_4_iProbe_2_bucketMinSize_10_bucketScale_5_qProbe_12.txt"
    cwd = os.getcwd()
    (tmp_path / "ref").mkdir()
    (tmp_path / "gpu").mkdir()
    capfd.readouterr()
    try:
        os.chdir(tmp_path / "ref")
        ref = r.query(Q, 7, verbose=True)
        ref_out = capfd.readouterr().out
        os.chdir(tmp_path / "gpu")
        got = idx.query(np.transpose(Q), 7, verbose=True)
        got_out = capfd.readouterr().out
    finally:
        os.chdir(cwd)
    assert np.array_equal(ref, got)
    assert _stat_lines(ref_out) and _stat_lines(ref_out) == _stat_lines(got_out)
    assert (tmp_path / "ref" / fname).read_bytes() == (tmp_path / "gpu" / fname).read_bytes()
