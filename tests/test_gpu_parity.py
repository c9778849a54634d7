"""Bit-exact parity of the CUDA path (through the C ABI) with the oracle on
seeded inputs small enough for the oracle: random signs, centre, hash codes,
bucket tables, probed buckets, candidate sets, top-k ids and scores."""
import numpy as np
import pytest

from falconnpp_b200 import synth
from tests.helpers import build_both, compare_build, compare_query

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,d,L,D,minSize,alpha,iProbes", [
    (3000, 24, 4, 32, 20, 0.01, 1),
    (3000, 24, 4, 32, 20, 0.01, 3),
    (5000, 64, 6, 64, 5, 0.05, 2),
    (4000, 200, 3, 256, 50, 0.01, 3),
    (2000, 100, 5, 128, 10, 0.5, 4),
])
def test_small_mixture(n, d, L, D, minSize, alpha, iProbes):
    X = synth.mixture(n, d, n_centres=16, seed=0)
    Q = synth.mixture(40, d, n_centres=16, seed=1)
    o, g, codes, scores = build_both(X, L, D, minSize, alpha, iProbes)
    compare_build(o, g, codes, scores)
    for qp in (1, 5, 3 * L):
        compare_query(o, g, Q, 10, qp)


def test_p0_integer_ties():
    """Integer, sign-symmetric data: centring is exact in any order and many
    scores tie, which exercises every exact heap replay."""
    X = synth.p0_integer(2000, 32, xmax=7)
    Q = synth.p0_queries(30, 32, qmax=3)
    o, g, codes, scores = build_both(X, 5, 32, 10, 0.02, 3)
    compare_build(o, g, codes, scores)
    assert np.all(o.center() == 0)
    for qp in (2, 7, 40):
        compare_query(o, g, Q, 20, qp)
