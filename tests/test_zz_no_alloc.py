"""fpp_rerank_probes_noalloc: the allocation-free variant of the gather /
rerank / top-k stage, for callers that cannot call cudaMalloc
(latency-critical serving threads, whose cudaMalloc / cudaFree would
synchronise the device, and processes whose device memory belongs to another
allocator).

It is called through the C ABI with device buffers the test owns, twice in a
row (the second call sees the scratch the first one left behind), and must
return exactly what fpp_query returns for the same probes: the ids are
integers, so the tolerance is equality, as in every other parity test here.
This file is collected last so a failure here never hides another test.
"""
import ctypes

import numpy as np
import pytest

from falconnpp_b200 import capi, synth

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("qprobes,k", [(6, 10), (24, 20)])
def test_noalloc_matches_query(qprobes, k):
    import torch

    n, d = 20000, 100
    X = synth.mixture(n, d, n_centres=32, seed=0)
    Q = synth.mixture(300, d, n_centres=32, seed=1)
    g = capi.Index(n, d)
    g.set_index_param(8, 128, 30, 0.01, 3, 8, 42)
    g.build(X)
    g.set_qprobes(qprobes)
    ref = g.query_dump(Q, k, qprobes)
    expected = ref["topk"]
    assert np.array_equal(expected, g.query(Q, k))

    dq = torch.from_numpy(Q).cuda()
    dp = torch.from_numpy(ref["probes"].view(np.int32)).cuda()
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        out = torch.full((Q.shape[0], k), -7, dtype=torch.int32, device="cuda")
        rc = capi.lib().fpp_rerank_probes_noalloc(g.h, ctypes.c_void_p(dq.data_ptr()), Q.shape[0],
                                                  ctypes.c_void_p(dp.data_ptr()), qprobes, k,
                                                  ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(stream))
        assert rc == 0, capi.lib().fpp_last_error().decode()
        got = out.cpu().numpy()
        assert np.array_equal(got, expected), f"call {call}: rows differ {np.where((got != expected).any(1))[0][:5]}"
    g.close()


def test_noalloc_rejects_bad_sizes():
    import torch

    n, d = 2000, 16
    X = synth.mixture(n, d, n_centres=8, seed=0)
    g = capi.Index(n, d)
    g.set_index_param(2, 16, 10, 0.1, 1, 8, 1)
    g.build(X)
    dq = torch.zeros((4, d), device="cuda")
    dp = torch.zeros((4, 2), dtype=torch.int32, device="cuda")
    out = torch.zeros((4, 2000), dtype=torch.int32, device="cuda")
    rc = capi.lib().fpp_rerank_probes_noalloc(g.h, ctypes.c_void_p(dq.data_ptr()), 4, ctypes.c_void_p(dp.data_ptr()),
                                              2, 2000, ctypes.c_void_p(out.data_ptr()), None)
    assert rc == capi.FPP_ERR_INVALID_ARGUMENT
    assert b"n_neighbors" in capi.lib().fpp_last_error()
    g.close()


def test_noalloc_rejects_out_of_range_probe():
    # caller-supplied probes are checked on the device: an id past the
    # index's n_tables * 4 * n_proj^2 buckets is read as an empty bucket and
    # the call reports it; the other queries' rows are still those of the
    # same probes without the bad id
    import torch

    n, d, k, qprobes = 5000, 32, 5, 4
    X = synth.mixture(n, d, n_centres=8, seed=0)
    Q = synth.mixture(16, d, n_centres=8, seed=1)
    g = capi.Index(n, d)
    g.set_index_param(4, 32, 10, 0.05, 2, 8, 3)
    g.build(X)
    g.set_qprobes(qprobes)
    ref = g.query_dump(Q, k, qprobes)
    probes = ref["probes"].copy()
    nb = g.info()["n_buckets"]
    probes[3, 1] = nb  # one past the last bucket
    probes[7, 0] = 0xFFFFFFF0
    dq = torch.from_numpy(Q).cuda()
    dp = torch.from_numpy(probes.view(np.int32)).cuda()
    out = torch.full((Q.shape[0], k), -7, dtype=torch.int32, device="cuda")
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = capi.lib().fpp_rerank_probes_noalloc(g.h, ctypes.c_void_p(dq.data_ptr()), Q.shape[0],
                                              ctypes.c_void_p(dp.data_ptr()), qprobes, k,
                                              ctypes.c_void_p(out.data_ptr()), stream)
    assert rc == capi.FPP_ERR_INVALID_ARGUMENT
    assert b"probe id" in capi.lib().fpp_last_error()
    got = out.cpu().numpy()
    good = [i for i in range(Q.shape[0]) if i not in (3, 7)]
    assert np.array_equal(got[good], ref["topk"][good])
    # the next call with valid probes succeeds (the status word is cleared)
    dp = torch.from_numpy(ref["probes"].view(np.int32)).cuda()
    rc = capi.lib().fpp_rerank_probes_noalloc(g.h, ctypes.c_void_p(dq.data_ptr()), Q.shape[0],
                                              ctypes.c_void_p(dp.data_ptr()), qprobes, k,
                                              ctypes.c_void_p(out.data_ptr()), stream)
    assert rc == 0, capi.lib().fpp_last_error().decode()
    assert np.array_equal(out.cpu().numpy(), ref["topk"])
    g.close()
