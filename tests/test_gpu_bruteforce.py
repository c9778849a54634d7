"""FP64 brute-force top-k on the GPU (the recall ground truth) against the
oracle's FP64 brute force (ties by ascending id) and against a torch FP64
reference at a larger size."""
import numpy as np
import pytest

from falconnpp_b200 import capi, synth
from oracle import oracle

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,d,nq,k", [(5000, 24, 37, 20), (20000, 200, 50, 100), (3000, 130, 9, 256)])
def test_bruteforce_matches_oracle(n, d, nq, k):
    import torch
    X = synth.mixture(n, d, n_centres=16, seed=0)
    Q = synth.mixture(nq, d, n_centres=16, seed=1)
    ref = oracle.bf_topk_f64(X, Q, k)
    dx = torch.from_numpy(X).cuda()
    dq = torch.from_numpy(Q).cuda()
    out = torch.zeros((nq, k), dtype=torch.int32, device="cuda")
    val = torch.zeros((nq, k), dtype=torch.float64, device="cuda")
    capi.bruteforce_topk_f64(dx.data_ptr(), n, d, dq.data_ptr(), nq, k, out.data_ptr(), val.data_ptr())
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy(), ref)
    exact = (torch.from_numpy(Q).double().cuda()[:, None, :] * dx.double()[out.long()]).sum(-1)
    assert torch.allclose(val, exact, rtol=1e-12, atol=1e-12)


def test_bruteforce_large_against_torch():
    import torch
    X = synth.mixture(1_000_000, 200, seed=0)
    Q = synth.mixture(64, 200, seed=1)
    dx = torch.from_numpy(X).cuda()
    dq = torch.from_numpy(Q).cuda()
    out = torch.zeros((64, 20), dtype=torch.int32, device="cuda")
    capi.bruteforce_topk_f64(dx.data_ptr(), X.shape[0], 200, dq.data_ptr(), 64, 20, out.data_ptr())
    torch.cuda.synchronize()
    sc = dq.double() @ dx.double().T
    ref = torch.topk(sc, 20, dim=1).indices.cpu().numpy()
    assert synth.recall_at_k(ref, out.cpu().numpy(), 20) == 1.0
