"""Shared helpers of the parity tests: run the same configuration through the
oracle and through the C ABI and compare every stage."""
from __future__ import annotations

import numpy as np

from falconnpp_b200 import capi
from oracle import oracle


def build_both(X, L, D, minSize, alpha, iProbes, seed=42, exact_order=True, dump_hash=True, threads=0):
    n, d = X.shape
    o = oracle.Index(n, d)
    o.set_index_param(L, D, minSize, alpha, iProbes, threads, seed)
    o.build(X)
    g = capi.Index(n, d)
    g.set_index_param(L, D, minSize, alpha, iProbes, 8, seed)
    g.set_option("exact_bucket_order", int(exact_order))
    codes = scores = None
    if dump_hash:
        codes, scores = g.build_dump_hash(X)
    else:
        g.build(X)
    return o, g, codes, scores


def compare_build(o, g, codes, scores, exact_order=True):
    """Bit-exact comparison of signs, centre, hash codes and bucket tables."""
    b1o, b2o = o.bits()
    b1g, b2g = g.dump_bits()
    assert np.array_equal(b1o, b1g) and np.array_equal(b2o, b2g), "random signs differ"
    assert np.array_equal(o.center().view(np.uint32), g.dump_center().view(np.uint32)), "centre differs"
    if codes is not None:
        co, so = o.hash_codes()
        assert np.array_equal(co, codes), f"hash codes differ at {np.argwhere(co != codes)[:5]}"
        assert np.array_equal(so.view(np.uint32), scores.view(np.uint32)), "hash scores differ"
    t = o.tables()
    start, ids = g.dump_tables()
    size_o = t["size"].astype(np.int64)
    size_g = np.diff(start.astype(np.int64))
    assert np.array_equal(size_o, size_g), "bucket sizes differ"
    assert len(ids) == len(t["ids"])
    if exact_order:
        assert np.array_equal(ids, t["ids"]), "bucket contents differ"
    else:
        # same kept set per bucket; order may differ only among equal scores
        so = np.repeat(np.arange(len(size_o)), size_o)
        ko = np.lexsort((t["ids"], so))
        kg = np.lexsort((ids, so))
        assert np.array_equal(t["ids"][ko], ids[kg]), "bucket sets differ"


def compare_query(o, g, Q, k, qprobes, check_cands=True):
    o.set_qprobes(qprobes)
    g.set_qprobes(qprobes)
    ro = o.query(Q, k, with_probes=True)
    cap = 0
    if check_cands:
        cap = int(max(1, ro["stats"][:, 1].max()))
    rg = g.query_dump(Q, k, qprobes, cand_cap=cap)
    # probed bucket sets
    po = np.sort(ro["probes"].astype(np.int64), axis=1)
    pg = np.sort(rg["probes"].astype(np.int64), axis=1)
    assert np.array_equal(po, pg), f"probe sets differ for queries {np.where((po != pg).any(1))[0][:5]}"
    assert np.array_equal(ro["stats"][:, 0], rg["stats"][:, 0]), "candidate counts differ"
    assert np.array_equal(ro["stats"][:, 1], rg["stats"][:, 1]), "unique candidate counts differ"
    if check_cands:
        for qi in range(Q.shape[0]):
            u = int(ro["stats"][qi, 1])
            cg = np.sort(rg["cands"][qi, :u])
            co = o.candidates(Q[qi])
            assert np.array_equal(co, cg), f"candidate set differs for query {qi}"
    assert np.array_equal(ro["topk"], rg["topk"]), \
        f"top-k ids differ for queries {np.where((ro['topk'] != rg['topk']).any(1))[0][:5]}"
    assert np.array_equal(ro["topk_val"].view(np.uint32), rg["topk_val"].view(np.uint32)), "top-k scores differ"
    return ro, rg
