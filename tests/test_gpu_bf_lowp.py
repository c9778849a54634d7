"""Brute-force block rerank in BF16 / FP8 on the tcgen05 tensor cores
(fpp_bruteforce_topk_lowp) against the FP64 exact top-k (the model of
BF::mips_topK, src/BF.cpp:17-86).

* Integer data whose BF16 copies are exact: every low-precision score equals
  the exact inner product, so the shortlist, the FP32 re-score and the
  returned ids must equal the FP64 top-k exactly (ties by ascending id).
  This pins the tensor-core pipeline itself (operand layout, swizzle, MMA
  shape, accumulator lanes and columns, the fused top-R).
* Mixture data: recall@k against FP64 >= 0.995 at shortlist 4k, the
  returned scores are the exact FP32 inner products of the returned ids
  (bit-identical to the query path's dot), and repeated calls agree.
* Ragged shapes: point and query counts that are not multiples of the
  128-row tiles.
* Crowded neighbours: points stored in increasing order of their inner
  product with one query, so that query's best rows all sit in the last row
  tile (one segment holds them all), with several query tiles per CTA range.
"""
import numpy as np
import pytest

from falconnpp_b200 import capi, synth

pytestmark = pytest.mark.gpu


def _index(X):
    g = capi.Index(*X.shape)
    g.set_index_param(2, 16 if X.shape[1] <= 16 else 64, 10, 0.1, 1, 8, 1)
    g.build(X)
    return g


def _lowp(g, Q, k, precision, mult):
    import torch
    dq = torch.from_numpy(np.ascontiguousarray(Q)).cuda()
    out = torch.full((len(Q), k), -9, dtype=torch.int32, device="cuda")
    val = torch.zeros((len(Q), k), dtype=torch.float32, device="cuda")
    g.bruteforce_lowp(dq.data_ptr(), len(Q), k, precision, mult, out.data_ptr(), val.data_ptr(),
                      torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return out.cpu().numpy(), val.cpu().numpy()


def _fp64(X, Q, k):
    import torch
    dx = torch.from_numpy(X).cuda()
    dq = torch.from_numpy(np.ascontiguousarray(Q)).cuda()
    out = torch.zeros((len(Q), k), dtype=torch.int32, device="cuda")
    val = torch.zeros((len(Q), k), dtype=torch.float64, device="cuda")
    capi.bruteforce_topk_f64(dx.data_ptr(), X.shape[0], X.shape[1], dq.data_ptr(), len(Q), k, out.data_ptr(),
                             val.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return out.cpu().numpy(), val.cpu().numpy()


@pytest.mark.parametrize("n,d,nq", [(20000, 64, 300), (5000, 200, 130), (1000, 40, 7)])
def test_bf16_exact_on_integer_data(n, d, nq):
    X = synth.p0_integer(n, d, xmax=15)
    Q = synth.p0_queries(nq, d, qmax=7)
    g = _index(X)
    ids, val = _lowp(g, Q, 10, 1, 4)
    ref, ref_v = _fp64(X, Q, 10)
    assert np.array_equal(val.astype(np.float64), ref_v), "scores differ from the exact inner products"
    bad = np.where((ids != ref).any(1))[0]
    assert len(bad) == 0, f"ids differ for queries {bad[:5]}"
    g.close()


@pytest.mark.parametrize("precision", [1, 2])
def test_mixture_recall_and_exact_scores(precision):
    from oracle import oracle
    X = synth.mixture(60000, 200, seed=0)
    Q = synth.mixture(500, 200, seed=1)
    g = _index(X)
    ids, val = _lowp(g, Q, 10, precision, 4)
    ref, _ = _fp64(X, Q, 10)
    rec = synth.recall_at_k(ref, ids, 10)
    assert rec >= 0.995, rec
    _, Xc = oracle.center(X)
    for qi in range(0, len(Q), 25):
        for j in range(10):
            assert val[qi, j] == np.float32(oracle.dot(Q[qi], Xc[ids[qi, j]])), (qi, j)
    assert np.all(np.diff(val, axis=1) <= 0)
    ids2, val2 = _lowp(g, Q, 10, precision, 4)
    assert np.array_equal(ids, ids2) and np.array_equal(val, val2)
    g.close()


@pytest.mark.parametrize("precision", [1, 2])
def test_ragged_shapes(precision):
    X = synth.mixture(1000 * 13 + 37, 100, n_centres=16, seed=0)
    Q = synth.mixture(129, 100, n_centres=16, seed=1)
    g = _index(X)
    ids, _ = _lowp(g, Q, 5, precision, 2)
    ref, _ = _fp64(X, Q, 5)
    assert synth.recall_at_k(ref, ids, 5) >= 0.99
    assert ids.min() >= 0 and ids.max() < X.shape[0]
    g.close()


@pytest.mark.parametrize("precision", [1, 2])
def test_crowded_neighbours(precision):
    X = synth.mixture(30000, 64, n_centres=16, seed=0)
    Q = synth.mixture(300, 64, n_centres=16, seed=1)
    X = np.ascontiguousarray(X[np.argsort(X @ Q[0], kind="stable")])
    g = _index(X)
    ids, val = _lowp(g, Q, 10, precision, 4)
    ref, _ = _fp64(X, Q, 10)
    assert synth.recall_at_k(ref, ids, 10) >= 0.99
    # query 0's top 10 are the last ten ids, in one row tile
    assert set(ref[0]) <= set(range(len(X) - 128, len(X)))
    assert synth.recall_at_k(ref[:1], ids[:1], 10) >= 0.9
    assert np.all(np.diff(val, axis=1) <= 0)
    g.close()


@pytest.mark.parametrize("nq", [1, 5, 129])
def test_few_queries_many_rows(nq):
    # one query tile against 1,563 row tiles: the units grow so that the
    # tile's segments fit the merge
    X = synth.mixture(200_000, 64, n_centres=32, seed=0)
    Q = synth.mixture(nq, 64, n_centres=32, seed=1)
    g = _index(X)
    ids, val = _lowp(g, Q, 10, 1, 4)
    ref, _ = _fp64(X, Q, 10)
    assert synth.recall_at_k(ref, ids, 10) >= 0.99
    assert np.all(np.diff(val, axis=1) <= 0)
    g.close()


def test_rejections():
    X = synth.mixture(2000, 64, n_centres=4, seed=0)
    g = _index(X)
    import torch
    dq = torch.zeros((4, 64), device="cuda")
    out = torch.zeros((4, 300), dtype=torch.int32, device="cuda")
    for args in [(4, 10, 0, 2), (4, 10, 3, 2), (4, 200, 1, 2), (4, 0, 1, 2)]:
        with pytest.raises(capi.FppError) as e:
            g.bruteforce_lowp(dq.data_ptr(), args[0], args[1], args[2], args[3], out.data_ptr())
        assert e.value.code == -1
    g.close()
