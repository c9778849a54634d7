"""ctypes wrappers of the CPU checkers: the oracle (oracle/falconnpp_oracle.cpp,
a restatement of the reference's algorithm) and the reference's own code
compiled from its sources (oracle/_ref/libfalconnpp_ref.so: src/FalconnPP.cpp,
src/Utilities.cpp and src/fht.c unchanged, against the Eigen / Boost subset in
oracle/shim/, through oracle/ref_harness.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU legs of bench.py, never by the product.  ``build()`` compiles the oracle
and, when the reference tree is present, the oracle/_ref libraries, with the
Makefile beside this file.  The reference tree is taken from the environment
variable FPP_REFERENCE_ROOT when it is set, else the Makefile's default.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liboracle.so")
REF_FHT = os.path.join(HERE, "_ref", "libfht_ref.so")
REF_LIB = os.path.join(HERE, "_ref", "libfalconnpp_ref.so")

_lib = None
_ref_lib = None


def _make_args() -> list[str]:
    root = os.environ.get("FPP_REFERENCE_ROOT")
    return [f"REF={root}"] if root else []


def build(force: bool = False) -> None:
    """Compile the oracle, and the oracle/_ref libraries where the reference
    tree is present (make decides from the sources' timestamps)."""
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(
            os.path.join(HERE, "falconnpp_oracle.cpp")):
        subprocess.run(["make", "-C", HERE, "-B" if force else "-s", LIB if not force else "all",
                        *_make_args()], check=True, capture_output=True)
    subprocess.run(["make", "-C", HERE, "-s", "ref", *_make_args()], check=True, capture_output=True)


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = ctypes.CDLL(LIB)
        vp, i32, i64, f32 = ctypes.c_void_p, ctypes.c_int, ctypes.c_longlong, ctypes.c_float
        sig = {
            "orc_fwht": (i32, [vp, i32]),
            "orc_dot": (f32, [vp, vp, i32]),
            "orc_hd3_bits": (None, [i64, i32, vp, vp]),
            "orc_center": (None, [vp, i64, i32, vp, vp]),
            "orc_create": (vp, [i32, i32]),
            "orc_destroy": (None, [vp]),
            "orc_set_index_param": (i32, [vp, i32, i32, i32, f32, i32, i32, i64]),
            "orc_set_qprobes": (None, [vp, i32]),
            "orc_set_threads": (None, [vp, i32]),
            "orc_build": (i64, [vp, vp]),
            "orc_get_center": (None, [vp, vp]),
            "orc_get_bits": (None, [vp, vp, vp]),
            "orc_get_hash": (None, [vp, vp, vp]),
            "orc_get_tables": (None, [vp, vp, vp, vp, vp, vp]),
            "orc_query": (i32, [vp, vp, i32, i32, vp, vp, vp, vp, vp]),
            "orc_query_candidates": (i64, [vp, vp, vp, i64]),
            "orc_bf_topk_f64": (None, [vp, i64, i32, vp, i32, i32, i32, vp]),
            "orc_import": (None, [vp, vp, vp, vp, vp, vp, vp, i64]),
            "orc_set_table_range": (None, [vp, i32, i32]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def ref_fht() -> ctypes.CDLL | None:
    """The reference's own fht_float (compiled from its sources), if built."""
    if not os.path.exists(REF_FHT):
        return None
    L = ctypes.CDLL(REF_FHT)
    L.fht_float.restype = ctypes.c_int
    L.fht_float.argtypes = [ctypes.c_void_p, ctypes.c_int]
    return L


def _p(a):
    return None if a is None else a.ctypes.data


def fwht(x: np.ndarray) -> np.ndarray:
    y = np.array(x, dtype=np.float32, copy=True)
    log_n = int(np.log2(y.size))
    lib().orc_fwht(_p(y), log_n)
    return y


def dot(q: np.ndarray, x: np.ndarray) -> float:
    q = np.ascontiguousarray(q, np.float32)
    x = np.ascontiguousarray(x, np.float32)
    return float(lib().orc_dot(_p(q), _p(x), q.size))


def hd3_bits(seed: int, nbits: int):
    b1 = np.zeros(nbits, np.uint8)
    b2 = np.zeros(nbits, np.uint8)
    lib().orc_hd3_bits(seed, nbits, _p(b1), _p(b2))
    return b1, b2


def center(X: np.ndarray):
    X = np.ascontiguousarray(X, np.float32)
    mean = np.zeros(X.shape[1], np.float32)
    Xc = np.zeros_like(X)
    lib().orc_center(_p(X), X.shape[0], X.shape[1], _p(mean), _p(Xc))
    return mean, Xc


def bf_topk_f64(X: np.ndarray, Q: np.ndarray, k: int, threads: int = 0) -> np.ndarray:
    X = np.ascontiguousarray(X, np.float32)
    Q = np.ascontiguousarray(Q, np.float32)
    out = np.zeros((Q.shape[0], k), np.int32)
    lib().orc_bf_topk_f64(_p(X), X.shape[0], X.shape[1], _p(Q), Q.shape[0], k, threads, _p(out))
    return out


class Index:
    """CPU restatement of the reference index (same parameters and outputs)."""

    def __init__(self, n: int, d: int):
        self.n, self.d = n, d
        self.h = lib().orc_create(n, d)

    def __del__(self):
        try:
            lib().orc_destroy(self.h)
        except Exception:
            pass

    def set_index_param(self, L, D, minSize, alpha, iProbes, threads=0, seed=-1):
        self.fht = lib().orc_set_index_param(self.h, L, D, minSize, alpha, iProbes, threads, seed)
        self.L, self.D, self.iProbes = L, D, iProbes

    def set_qprobes(self, q):
        self.qProbes = q
        lib().orc_set_qprobes(self.h, q)

    def set_table_range(self, lo, hi):
        lib().orc_set_table_range(self.h, lo, hi)

    def set_threads(self, t):
        lib().orc_set_threads(self.h, t)

    def build(self, X: np.ndarray) -> int:
        X = np.ascontiguousarray(X, np.float32)
        self.n_ids = int(lib().orc_build(self.h, _p(X)))
        return self.n_ids

    def import_index(self, Xc, center, b1, b2, start, ids):
        """Adopt an index built elsewhere (e.g. dumped from the GPU)."""
        self._keep = [np.ascontiguousarray(a) for a in (Xc, center, b1, b2)]
        start = np.ascontiguousarray(start, np.uint32)
        ids = np.ascontiguousarray(ids, np.int32)
        lib().orc_import(self.h, _p(self._keep[0]), _p(self._keep[1]), _p(self._keep[2]), _p(self._keep[3]),
                         _p(start), _p(ids), len(ids))
        self.n_ids = len(ids)

    def center(self):
        c = np.zeros(self.d, np.float32)
        lib().orc_get_center(self.h, _p(c))
        return c

    def bits(self):
        nbits = self.L * 3 * self.fht
        b1 = np.zeros(nbits, np.uint8)
        b2 = np.zeros(nbits, np.uint8)
        lib().orc_get_bits(self.h, _p(b1), _p(b2))
        return b1, b2

    def hash_codes(self):
        codes = np.zeros((self.L, self.n, self.iProbes), np.int32)
        scores = np.zeros((self.L, self.n, self.iProbes), np.float32)
        lib().orc_get_hash(self.h, _p(codes), _p(scores))
        return codes, scores

    def tables(self):
        nb = self.L * 4 * self.D * self.D
        start = np.zeros(nb + 1, np.uint64)
        size = np.zeros(nb, np.uint16)
        raw = np.zeros(nb, np.uint32)
        ids = np.zeros(max(1, self.n_ids), np.int32)
        sc = np.zeros(max(1, self.n_ids), np.float32)
        lib().orc_get_tables(self.h, _p(start), _p(size), _p(raw), _p(ids), _p(sc))
        return dict(start=start, size=size, raw=raw, ids=ids[: self.n_ids], scores=sc[: self.n_ids])

    def query(self, Q: np.ndarray, k: int, with_probes: bool = False):
        Q = np.ascontiguousarray(Q, np.float32)
        nq = Q.shape[0]
        out = np.zeros((nq, k), np.int32)
        val = np.zeros((nq, k), np.float32)
        stats = np.zeros((nq, 4), np.int64)
        probes = np.zeros((nq, self.qProbes), np.int32) if with_probes else None
        pval = np.zeros((nq, self.qProbes), np.float32) if with_probes else None
        rc = lib().orc_query(self.h, _p(Q), nq, k, _p(out), _p(val), _p(probes), _p(pval), _p(stats))
        if rc != 0:
            raise ValueError("oracle query: qProbes too large for n_proj")
        return dict(topk=out, topk_val=val, stats=stats, probes=probes, probe_val=pval)

    def candidates(self, q: np.ndarray) -> np.ndarray:
        q = np.ascontiguousarray(q, np.float32)
        cap = self.n
        out = np.zeros(cap, np.int32)
        c = int(lib().orc_query_candidates(self.h, _p(q), _p(out), cap))
        return out[:c]


def ref_lib() -> ctypes.CDLL | None:
    """The reference's own FalconnPP code (compiled from its sources), if built."""
    global _ref_lib
    if _ref_lib is None:
        if not os.path.exists(REF_LIB):
            return None
        L = ctypes.CDLL(REF_LIB)
        vp, i32, i64, f32 = ctypes.c_void_p, ctypes.c_int, ctypes.c_longlong, ctypes.c_float
        sig = {
            "ref_create": (vp, [i32, i32]),
            "ref_destroy": (None, [vp]),
            "ref_set_index_param": (None, [vp, i32, i32, i32, f32, i32, i32, i32]),
            "ref_set_qprobes": (None, [vp, i32]),
            "ref_set_threads": (None, [vp, i32]),
            "ref_build": (None, [vp, vp, i32]),
            "ref_query": (None, [vp, vp, i32, i32, i32, i32, vp]),
            "ref_import": (None, [vp, vp, vp, vp, i64, vp, i64, vp, i64]),
            "ref_fht_dim": (i32, [vp]),
            "ref_num_ids": (i64, [vp]),
            "ref_num_buckets": (i64, [vp]),
            "ref_get_tables": (None, [vp, vp, vp, vp]),
            "ref_num_ids_2d": (i64, [vp]),
            "ref_get_tables_2d": (None, [vp, vp, vp]),
            "ref_get_centered": (None, [vp, vp]),
            "ref_get_bits": (None, [vp, vp, vp]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _ref_lib = L
    return _ref_lib


class Reference:
    """The reference's FalconnPP class itself (src/FalconnPP.h:10-132), built
    from its own sources: setIndexParam / build / set_qProbes / query, and
    the 2D build2D / query2D, plus reads of its index internals."""

    def __init__(self, n: int, d: int):
        L = ref_lib()
        if L is None:
            raise RuntimeError("oracle/_ref/libfalconnpp_ref.so is not built (the reference tree is absent)")
        self.n, self.d = n, d
        self.h = L.ref_create(n, d)
        self.two_d = False

    def __del__(self):
        try:
            ref_lib().ref_destroy(self.h)
        except Exception:
            pass

    def set_index_param(self, L, D, minSize, alpha, iProbes, threads=0, seed=-1):
        ref_lib().ref_set_index_param(self.h, L, D, minSize, alpha, iProbes, threads, seed)
        self.L, self.D, self.iProbes = L, D, iProbes
        self.fht = int(ref_lib().ref_fht_dim(self.h))

    def set_qprobes(self, q):
        self.qProbes = q
        ref_lib().ref_set_qprobes(self.h, q)

    def set_threads(self, t):
        ref_lib().ref_set_threads(self.h, t)

    def build(self, X: np.ndarray, two_d: bool = False):
        self._X = np.ascontiguousarray(X, np.float32)
        self.two_d = two_d
        ref_lib().ref_build(self.h, _p(self._X), int(two_d))

    def query(self, Q: np.ndarray, k: int, verbose: bool = False) -> np.ndarray:
        Q = np.ascontiguousarray(Q, np.float32)
        out = np.zeros((Q.shape[0], k), np.int32)
        ref_lib().ref_query(self.h, _p(Q), Q.shape[0], k, int(verbose), int(self.two_d), _p(out))
        return out

    def bits(self):
        nbits = self.L * 3 * self.fht
        b1 = np.zeros(nbits, np.uint8)
        b2 = np.zeros(nbits, np.uint8)
        ref_lib().ref_get_bits(self.h, _p(b1), _p(b2))
        return b1, b2

    def import_index(self, Xc, b1, b2, start, ids):
        """Adopt an index built elsewhere (dumped from the GPU): its queries
        then run through the reference's own query2Layers_1D."""
        Xc = np.ascontiguousarray(Xc, np.float32)
        b1 = np.ascontiguousarray(b1, np.uint8)
        b2 = np.ascontiguousarray(b2, np.uint8)
        start = np.ascontiguousarray(start, np.uint32)
        ids = np.ascontiguousarray(ids, np.int32)
        if np.diff(start.astype(np.int64)).max(initial=0) > 65535:
            raise ValueError("a bucket holds more than 65535 ids (the reference's uint16 size)")
        ref_lib().ref_import(self.h, _p(Xc), _p(b1), _p(b2), b1.size, _p(start), start.size - 1, _p(ids), ids.size)
        self.two_d = False

    def centered(self) -> np.ndarray:
        Xc = np.zeros((self.n, self.d), np.float32)
        ref_lib().ref_get_centered(self.h, _p(Xc))
        return Xc

    def buckets(self):
        """Per bucket (global id l * 4D^2 + h): the reference's ids in its
        stored order.  Returns (sizes, ids concatenated in bucket order)."""
        L = ref_lib()
        if self.two_d:
            nb = self.L * 4 * self.D * self.D
            size = np.zeros(nb, np.uint32)
            ids = np.zeros(max(1, int(L.ref_num_ids_2d(self.h))), np.int32)
            L.ref_get_tables_2d(self.h, _p(size), _p(ids))
            return size.astype(np.int64), ids[: int(size.sum())]
        nb = int(L.ref_num_buckets(self.h))
        pos = np.zeros(nb, np.uint32)
        size = np.zeros(nb, np.uint16)
        raw = np.zeros(max(1, int(L.ref_num_ids(self.h))), np.int32)
        L.ref_get_tables(self.h, _p(pos), _p(size), _p(raw))
        size = size.astype(np.int64)
        # gather each bucket's range [pos, pos + size) into bucket order
        total = int(size.sum())
        starts = np.repeat(pos.astype(np.int64), size)
        within = np.arange(total, dtype=np.int64) - np.repeat(np.cumsum(size) - size, size)
        return size, raw[starts + within]
