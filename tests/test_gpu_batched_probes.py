"""The low-precision batched forms hash exactly like the reference.

BF16 and FP8 change only the candidate rerank.  The rotation, the
cross-polytope hash, the per-table probe lists and the global probe cut stay
the reference's FP32 arithmetic (src/FalconnPP.cpp:358-582), so every batched
form must probe the same buckets and gather the same candidates as the plain
FP32 path, which the parity tests pin to the oracle.  Checked per query,
exactly: the probed bucket set, the candidate count and the unique-candidate
count, on the 100k x 200 configuration (fhtDim 256, one and two probes per
table) and on integer tie-heavy data (P0), where the plain path is also
compared with the oracle directly.
"""
import numpy as np
import pytest

from falconnpp_b200 import capi, synth
from tests.helpers import build_both, compare_query

pytestmark = pytest.mark.gpu


def _batched_dump(g, Q, k, qp, precision):
    import torch
    g.set_query_form(1, precision, 4)
    g.set_qprobes(qp)
    dq = torch.from_numpy(np.ascontiguousarray(Q)).cuda()
    nq = len(Q)
    out = torch.full((nq, k), -9, dtype=torch.int32, device="cuda")
    probes = torch.zeros((nq, qp), dtype=torch.int32, device="cuda")
    counts = torch.zeros((nq, 2), dtype=torch.int32, device="cuda")
    s = torch.cuda.Stream()
    g.query_batched_dump(dq.data_ptr(), nq, k, out.data_ptr(), None, probes.data_ptr(), counts.data_ptr(),
                         s.cuda_stream)
    torch.cuda.synchronize()
    g.set_query_form(0, 0, 4)
    return out.cpu().numpy(), probes.cpu().numpy().view(np.uint32), counts.cpu().numpy().astype(np.int64)


def _check_same_probes(g, Q, k, qp, precisions=(0, 1, 2)):
    g.set_query_form(0, 0, 4)
    g.set_qprobes(qp)
    plain = g.query_dump(Q, k, qp)
    po = np.sort(plain["probes"].astype(np.int64), axis=1)
    for prec in precisions:
        ids, probes, counts = _batched_dump(g, Q, k, qp, prec)
        pb = np.sort(probes.astype(np.int64), axis=1)
        bad = np.where((po != pb).any(1))[0]
        assert len(bad) == 0, f"precision {prec}, qProbes {qp}: probe sets differ for queries {bad[:5]}"
        assert np.array_equal(counts[:, 0], plain["stats"][:, 0]), f"precision {prec}: candidate counts differ"
        assert np.array_equal(counts[:, 1], plain["stats"][:, 1]), f"precision {prec}: unique counts differ"
        if prec == 0:
            assert np.array_equal(ids, plain["topk"]), "FP32 batched top-k differs from the plain path"
    return plain


def test_cfg1_probes_equal_plain():
    # 100k x 200 mixture, L=50, n_proj=256 (fhtDim 256), iProbes=1: qProbes 10
    # keeps one probe per table (the regime the opt-in tensor-core rotation
    # would take), 40 keeps two
    X = synth.mixture(100_000, 200, n_centres=256, norm_sigma=0.4, seed=0)
    Q = synth.mixture(1000, 200, n_centres=256, norm_sigma=0.4, seed=1)
    g = capi.Index(*X.shape)
    g.set_index_param(50, 256, 500, 0.01, 1, 8, 42)
    g.build(X)
    for qp in (10, 40):
        _check_same_probes(g, Q, 20, qp)
    g.close()


def test_p0_probes_equal_oracle_and_plain():
    # integer sign-symmetric data at fhtDim 256: rotated coordinates and
    # bucket scores tie often, so any deviation from the FP32 hash shows
    X = synth.p0_integer(4000, 200, xmax=15)
    Q = synth.p0_queries(80, 200, qmax=3)
    o, g, _, _ = build_both(X, 8, 256, 20, 0.02, 3, dump_hash=False)
    for qp in (4, 16):
        compare_query(o, g, Q, 20, qp, check_cands=False)
        _check_same_probes(g, Q, 20, qp)
    g.close()


def test_tc_rotation_is_opt_in():
    # the default hashes in FP32: turning the opt-in tensor-core rotation on
    # and off again restores the exact probes
    X = synth.mixture(20_000, 200, seed=0)
    Q = synth.mixture(200, 200, seed=1)
    g = capi.Index(*X.shape)
    g.set_index_param(20, 256, 50, 0.01, 3, 8, 42)
    g.build(X)
    _check_same_probes(g, Q, 10, 8, precisions=(2,))
    g.set_option("tc_rotation", 1)
    g.set_option("tc_rotation", 0)
    _check_same_probes(g, Q, 10, 8, precisions=(1, 2))
    g.close()
