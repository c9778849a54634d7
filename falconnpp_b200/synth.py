"""Seeded synthetic MIPS data: Gaussian-mixture points with log-normal norms.

The reference measures on Glove200 / NYTimes / Glove300, none of which is
available here; these generators stand in for them with the shapes and value
distributions of the benchmark configurations:

* mixture centres ~ N(0, I) in d dimensions, ``n_centres`` of them;
* a point = its centre + ``sigma`` * N(0, I) (``sigma`` = 0.3);
* the point is scaled to unit norm and then multiplied by a log-normal factor
  exp(N(0, ``norm_sigma``)), so norms vary and the search is unnormalised MIPS.

Data and queries come from numpy's PCG64 with separate seeds (data 0, queries
1 by default); queries are held out (drawn independently from the same mixture).
Everything is float32, point-major (n x d), which is the memory layout of the
reference's d x n column-major input matrix.
"""
from __future__ import annotations

import numpy as np


def mixture(n: int, d: int, n_centres: int = 256, sigma: float = 0.3, norm_sigma: float = 0.4,
            seed: int = 0, centre_seed: int = 12345, chunk: int = 1 << 18) -> np.ndarray:
    """n x d float32 points from the mixture described in the module docstring."""
    crng = np.random.Generator(np.random.PCG64(centre_seed))
    centres = crng.standard_normal((n_centres, d)).astype(np.float32)
    rng = np.random.Generator(np.random.PCG64(seed))
    out = np.empty((n, d), dtype=np.float32)
    for s in range(0, n, chunk):
        e = min(n, s + chunk)
        m = e - s
        lab = rng.integers(0, n_centres, size=m)
        x = centres[lab] + np.float32(sigma) * rng.standard_normal((m, d), dtype=np.float32)
        nrm = np.linalg.norm(x, axis=1, keepdims=True)
        nrm[nrm == 0] = 1.0
        scale = np.exp(rng.normal(0.0, norm_sigma, size=(m, 1))).astype(np.float32)
        out[s:e] = (x / nrm * scale).astype(np.float32)
    return out


def p0_integer(n: int, d: int, xmax: int = 1023, seed: int = 7) -> np.ndarray:
    """Integer-valued, sign-symmetric data (each x is paired with -x).

    Per-dimension sums are exactly zero in any order, so the centring mean is
    exactly 0 whatever the summation order, and with |q| small enough every dot
    product is an exact integer.  n must be even.
    """
    assert n % 2 == 0
    rng = np.random.Generator(np.random.PCG64(seed))
    half = rng.integers(-xmax, xmax + 1, size=(n // 2, d)).astype(np.float32)
    out = np.empty((n, d), dtype=np.float32)
    out[0::2] = half
    out[1::2] = -half
    return out


def p0_queries(nq: int, d: int, qmax: int = 63, seed: int = 8) -> np.ndarray:
    rng = np.random.Generator(np.random.PCG64(seed))
    return rng.integers(-qmax, qmax + 1, size=(nq, d)).astype(np.float32)


def recall_at_k(truth: np.ndarray, answer: np.ndarray, k: int) -> float:
    """Mean |truth[:k] & answer| / k over queries (test/falconnpp.py:180-186)."""
    score = 0.0
    for t, a in zip(truth, answer):
        score += len(set(t[:k].tolist()).intersection(set(a.tolist()))) / k
    return score / len(truth)
