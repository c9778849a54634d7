"""Regenerates the committed fixtures in tests/golden/ (run from the repo root:
``python tests/golden/make_golden.py``).

* fwht_kat.npz     — inputs and outputs of the reference's own fht_float
                     (src/fht.c compiled from the reference sources into
                     oracle/_ref/libfht_ref.so by oracle/Makefile): one
                     transform and three chained transforms, log_n = 1..10.
                     This pins the FWHT without the reference tree present.
* rng_bits.npz     — bitHD1/bitHD2 streams of src/FalconnPP.h:52-68 (libstdc++
                     default_random_engine + uniform_int_distribution) for a
                     few seeds, as produced by the oracle.
* small_index.npz  — a tiny index (inputs, centre, hash codes, CSR tables,
                     top-k of a few queries) from the oracle: a regression
                     fixture for the oracle and a parity fixture for the GPU.
* p0_index.npz     — the same on integer, sign-symmetric data (P0), where the
                     centre is exactly 0 and every dot product is exact.
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from falconnpp_b200 import synth  # noqa: E402
from oracle import oracle  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def fwht_kat():
    ref = oracle.ref_fht()
    if ref is None:
        raise SystemExit("oracle/_ref/libfht_ref.so missing: run `make -C oracle` with the reference tree present")
    rng = np.random.Generator(np.random.PCG64(2024))
    xs, y1, y3, logn = [], [], [], []
    for log_n in range(1, 11):
        for t in range(4):
            x = (rng.standard_normal(1 << log_n) * rng.uniform(0.01, 100)).astype(np.float32)
            a = x.copy()
            ref.fht_float(a.ctypes.data, log_n)
            b = a.copy()
            ref.fht_float(b.ctypes.data, log_n)
            ref.fht_float(b.ctypes.data, log_n)
            xs.append(np.pad(x, (0, 1024 - x.size)))
            y1.append(np.pad(a, (0, 1024 - a.size)))
            y3.append(np.pad(b, (0, 1024 - b.size)))
            logn.append(log_n)
    np.savez_compressed(os.path.join(OUT, "fwht_kat.npz"), x=np.array(xs), y1=np.array(y1), y3=np.array(y3),
                        log_n=np.array(logn, np.int32))


def rng_bits():
    seeds = [0, 1, 42, 12345, 2 ** 31 - 1]
    out = {}
    for s in seeds:
        b1, b2 = oracle.hd3_bits(s, 3 * 64 * 5)
        out[f"b1_{s}"] = b1
        out[f"b2_{s}"] = b2
    np.savez_compressed(os.path.join(OUT, "rng_bits.npz"), seeds=np.array(seeds, np.int64), **out)


def index_fixture(name, X, Q, L, D, minSize, alpha, iProbes, qprobes, k):
    n, d = X.shape
    o = oracle.Index(n, d)
    o.set_index_param(L, D, minSize, alpha, iProbes, 1, 42)
    o.build(X)
    codes, scores = o.hash_codes()
    t = o.tables()
    o.set_qprobes(qprobes)
    r = o.query(Q, k, with_probes=True)
    np.savez_compressed(os.path.join(OUT, name), X=X, Q=Q,
                        params=np.array([L, D, minSize, iProbes, qprobes, k], np.int64),
                        alpha=np.float32(alpha), center=o.center(), codes=codes, scores=scores,
                        start=t["start"], size=t["size"], ids=t["ids"], topk=r["topk"], topk_val=r["topk_val"],
                        probes=r["probes"], stats=r["stats"])


if __name__ == "__main__":
    oracle.build()
    fwht_kat()
    rng_bits()
    X = synth.mixture(600, 20, n_centres=6, seed=3)
    Q = synth.mixture(12, 20, n_centres=6, seed=4)
    index_fixture("small_index.npz", X, Q, 3, 16, 8, 0.05, 2, 4, 5)
    Xp = synth.p0_integer(400, 12, xmax=5)
    Qp = synth.p0_queries(10, 12, qmax=3)
    index_fixture("p0_index.npz", Xp, Qp, 4, 8, 4, 0.1, 2, 6, 8)
    print("fixtures written to", OUT)
