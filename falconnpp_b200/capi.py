"""ctypes view of the C ABI in include/falconnpp_b200.h.

Used by the tests and the benchmark to call the library exactly as a foreign
caller (cgo, JNI, another C program) would: plain pointers and sizes.
``Index`` wraps one handle and raises ``FppError`` on a negative status.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import LIBRARY_PATH, _require_native

# Every symbol the header declares (tests check the library exports them all).
EXPORTED = [
    "fpp_create", "fpp_destroy", "fpp_set_index_param", "fpp_set_qprobes", "fpp_set_threads", "fpp_clear",
    "fpp_build", "fpp_build_device", "fpp_query", "fpp_query_device", "fpp_last_error", "fpp_get_info",
    "fpp_get_stats", "fpp_set_option", "fpp_print_build_report", "fpp_dump_bits", "fpp_dump_center",
    "fpp_dump_tables", "fpp_build_dump_hash", "fpp_query_dump", "fpp_rerank_probes_noalloc",
    "fpp_set_query_form", "fpp_query_batched", "fpp_query_batched_dump", "fpp_autotune",
    "fpp_server_create", "fpp_server_submit", "fpp_server_wait", "fpp_server_stats", "fpp_server_destroy",
    "fpp_bruteforce_topk_f64", "fpp_bruteforce_topk_lowp", "fpp_save", "fpp_load", "fpp_load_txt", "fpp_output_file",
]

_lib = None
FPP_ERR_INVALID_ARGUMENT = -1


class FppError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        _require_native()
        L = ctypes.CDLL(LIBRARY_PATH)
        vp, i32, i64, f32 = ctypes.c_void_p, ctypes.c_int, ctypes.c_longlong, ctypes.c_float
        sig = {
            "fpp_create": (i32, [i32, i32, ctypes.POINTER(vp)]),
            "fpp_destroy": (None, [vp]),
            "fpp_set_index_param": (i32, [vp, i32, i32, i32, f32, i32, i32, i32]),
            "fpp_set_qprobes": (i32, [vp, i32]),
            "fpp_set_threads": (i32, [vp, i32]),
            "fpp_clear": (i32, [vp]),
            "fpp_build": (i32, [vp, vp]),
            "fpp_build_device": (i32, [vp, vp, vp]),
            "fpp_query": (i32, [vp, vp, i32, i32, i32, vp]),
            "fpp_query_device": (i32, [vp, vp, i32, i32, vp, vp]),
            "fpp_last_error": (ctypes.c_char_p, []),
            "fpp_get_info": (i32, [vp, vp, i32]),
            "fpp_get_stats": (i32, [vp, i32, vp, i32]),
            "fpp_set_option": (i32, [vp, ctypes.c_char_p, i64]),
            "fpp_print_build_report": (None, [vp]),
            "fpp_dump_bits": (i32, [vp, vp, vp]),
            "fpp_dump_center": (i32, [vp, vp]),
            "fpp_dump_tables": (i32, [vp, vp, vp]),
            "fpp_build_dump_hash": (i32, [vp, vp, vp, vp]),
            "fpp_query_dump": (i32, [vp, vp, i32, i32, vp, vp, vp, vp, vp, vp, i64]),
            "fpp_rerank_probes_noalloc": (i32, [vp, vp, i32, vp, i32, i32, vp, vp]),
            "fpp_set_query_form": (i32, [vp, i32, i32, i32]),
            "fpp_query_batched": (i32, [vp, vp, i32, vp, vp, i32, i32, vp, i32, vp, vp]),
            "fpp_query_batched_dump": (i32, [vp, vp, i32, i32, vp, vp, vp, vp, vp]),
            "fpp_autotune": (i32, [vp, vp, i32, i32, ctypes.c_double, vp, vp]),
            "fpp_server_create": (i32, [vp, i32, i64, i32, i32, i32, ctypes.POINTER(vp)]),
            "fpp_server_submit": (i32, [vp, vp, i32, i32, i32, vp, ctypes.POINTER(i64)]),
            "fpp_server_wait": (i32, [vp, i64, ctypes.POINTER(ctypes.c_double)]),
            "fpp_server_stats": (i32, [vp, vp, i32]),
            "fpp_server_destroy": (None, [vp]),
            "fpp_bruteforce_topk_f64": (i32, [vp, i64, i32, vp, i32, i32, vp, vp, vp]),
            "fpp_bruteforce_topk_lowp": (i32, [vp, vp, i32, i32, i32, i32, vp, vp, vp]),
            "fpp_save": (i32, [vp, ctypes.c_char_p]),
            "fpp_load": (i32, [vp, ctypes.c_char_p]),
            "fpp_load_txt": (i32, [ctypes.c_char_p, i32, i32, vp, vp]),
            "fpp_output_file": (i32, [ctypes.c_char_p, vp, i32, i32]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _check(rc: int) -> None:
    if rc != 0:
        raise FppError(rc, lib().fpp_last_error().decode())


def _ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data


class Index:
    """One index handle.  Points/queries are (n, d) float32 C-contiguous arrays
    (the memory layout of the reference's d x n column-major matrices)."""

    def __init__(self, n_points: int, n_features: int):
        self.n, self.d = n_points, n_features
        h = ctypes.c_void_p()
        _check(lib().fpp_create(n_points, n_features, ctypes.byref(h)))
        self.h = h

    def close(self):
        if self.h:
            lib().fpp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_index_param(self, n_tables, n_proj, bucket_minSize, bucket_scale, iProbes, n_threads=8, random_seed=-1):
        _check(lib().fpp_set_index_param(self.h, n_tables, n_proj, bucket_minSize, bucket_scale, iProbes, n_threads,
                                         random_seed))
        self.L, self.D, self.iProbes = n_tables, n_proj, iProbes

    def set_qprobes(self, q: int):
        _check(lib().fpp_set_qprobes(self.h, q))

    def clear(self):
        """The reference's clear() (src/FalconnPP.h:102-111): drops the index, keeps the parameters."""
        _check(lib().fpp_clear(self.h))

    def set_option(self, key: str, value: int):
        _check(lib().fpp_set_option(self.h, key.encode(), int(value)))

    def build(self, X: np.ndarray):
        X = np.ascontiguousarray(X, dtype=np.float32)
        assert X.shape == (self.n, self.d)
        _check(lib().fpp_build(self.h, _ptr(X)))

    def build_device(self, ptr: int, stream: int | None = None):
        _check(lib().fpp_build_device(self.h, ctypes.c_void_p(ptr), ctypes.c_void_p(stream or 0)))

    def build_dump_hash(self, X: np.ndarray):
        X = np.ascontiguousarray(X, dtype=np.float32)
        codes = np.zeros((self.L, self.n, self.iProbes), np.int32)
        scores = np.zeros((self.L, self.n, self.iProbes), np.float32)
        _check(lib().fpp_build_dump_hash(self.h, _ptr(X), _ptr(codes), _ptr(scores)))
        return codes, scores

    def query(self, Q: np.ndarray, k: int, verbose: bool = False) -> np.ndarray:
        Q = np.ascontiguousarray(Q, dtype=np.float32)
        out = np.zeros((Q.shape[0], k), np.int32)
        _check(lib().fpp_query(self.h, _ptr(Q), Q.shape[0], k, int(verbose), _ptr(out)))
        return out

    def query_device(self, q_ptr: int, nq: int, k: int, out_ptr: int, stream: int | None = None):
        _check(lib().fpp_query_device(self.h, ctypes.c_void_p(q_ptr), nq, k, ctypes.c_void_p(out_ptr),
                                      ctypes.c_void_p(stream or 0)))

    def query_dump(self, Q: np.ndarray, k: int, qprobes: int, cand_cap: int = 0):
        Q = np.ascontiguousarray(Q, dtype=np.float32)
        nq = Q.shape[0]
        out = np.zeros((nq, k), np.int32)
        val = np.zeros((nq, k), np.float32)
        probes = np.zeros((nq, qprobes), np.uint32)
        pval = np.zeros((nq, qprobes), np.float32)
        stats = np.zeros((nq, 4), np.int64)
        cands = np.full((nq, cand_cap), -1, np.int32) if cand_cap else None
        _check(lib().fpp_query_dump(self.h, _ptr(Q), nq, k, _ptr(out), _ptr(val), _ptr(probes), _ptr(pval),
                                    _ptr(stats), _ptr(cands), cand_cap))
        return dict(topk=out, topk_val=val, probes=probes, probe_val=pval, stats=stats, cands=cands)

    def set_query_form(self, form: int, precision: int = 0, shortlist_mult: int = 4):
        _check(lib().fpp_set_query_form(self.h, form, precision, shortlist_mult))

    def query_batched(self, q_ptr: int, nq: int, k_ptr: int | None, qp_ptr: int | None, k_max: int, qp_max: int,
                      out_ptr: int, out_stride: int, val_ptr: int | None = None, stream: int | None = None):
        _check(lib().fpp_query_batched(self.h, ctypes.c_void_p(q_ptr), nq, ctypes.c_void_p(k_ptr or 0),
                                       ctypes.c_void_p(qp_ptr or 0), k_max, qp_max, ctypes.c_void_p(out_ptr),
                                       out_stride, ctypes.c_void_p(val_ptr or 0), ctypes.c_void_p(stream or 0)))

    def query_batched_dump(self, q_ptr: int, nq: int, k: int, out_ptr: int, val_ptr: int | None,
                           probes_ptr: int | None, counts_ptr: int | None, stream: int | None = None):
        _check(lib().fpp_query_batched_dump(self.h, ctypes.c_void_p(q_ptr), nq, k, ctypes.c_void_p(out_ptr),
                                            ctypes.c_void_p(val_ptr or 0), ctypes.c_void_p(probes_ptr or 0),
                                            ctypes.c_void_p(counts_ptr or 0), ctypes.c_void_p(stream or 0)))

    def autotune(self, q_ptr: int, nq: int, k: int, min_agreement: float = 0.99, stream: int | None = None) -> dict:
        rep = np.zeros(8, np.float64)
        _check(lib().fpp_autotune(self.h, ctypes.c_void_p(q_ptr), nq, k, min_agreement, _ptr(rep),
                                  ctypes.c_void_p(stream or 0)))
        return dict(ms=rep[0], blocks_per_sm=int(rep[1]), precision=int(rep[2]), shortlist_mult=int(rep[3]),
                    agreement=rep[4], tried=int(rep[5]), split_hash=int(rep[6]), reorder=int(rep[7]))

    def bruteforce_lowp(self, q_ptr: int, nq: int, k: int, precision: int, shortlist_mult: int, out_ptr: int,
                        val_ptr: int | None = None, stream: int | None = None):
        _check(lib().fpp_bruteforce_topk_lowp(self.h, ctypes.c_void_p(q_ptr), nq, k, precision, shortlist_mult,
                                              ctypes.c_void_p(out_ptr), ctypes.c_void_p(val_ptr or 0),
                                              ctypes.c_void_p(stream or 0)))

    def info(self) -> dict:
        v = np.zeros(9, np.int64)
        _check(lib().fpp_get_info(self.h, _ptr(v), 9))
        return dict(fhtDim=int(v[0]), n_ids=int(v[1]), max_kept=int(v[2]), n_buckets=int(v[3]), built=bool(v[4]),
                    device=int(v[5]), n_tables=int(v[6]), n_proj=int(v[7]), iProbes=int(v[8]))

    def stats(self, kind: int) -> np.ndarray:
        v = np.zeros(11, np.float64)
        _check(lib().fpp_get_stats(self.h, kind, _ptr(v), 11))
        return v

    def dump_bits(self):
        info = self.info()
        nbits = info["n_tables"] * 3 * info["fhtDim"]
        b1 = np.zeros(nbits, np.uint8)
        b2 = np.zeros(nbits, np.uint8)
        _check(lib().fpp_dump_bits(self.h, _ptr(b1), _ptr(b2)))
        return b1, b2

    def dump_center(self):
        c = np.zeros(self.d, np.float32)
        _check(lib().fpp_dump_center(self.h, _ptr(c)))
        return c

    def save(self, path: str):
        _check(lib().fpp_save(self.h, os.fsencode(path)))

    def load(self, path: str):
        _check(lib().fpp_load(self.h, os.fsencode(path)))

    def dump_tables(self):
        info = self.info()
        start = np.zeros(info["n_buckets"] + 1, np.uint32)
        ids = np.zeros(max(1, info["n_ids"]), np.int32)
        _check(lib().fpp_dump_tables(self.h, _ptr(start), _ptr(ids)))
        return start, ids[: info["n_ids"]]


class Server:
    """Continuous-batching serving loop over an Index (fpp_server_*)."""

    def __init__(self, index: Index, n_streams=3, memory_budget=1 << 30, max_batch=8192, k_max=100,
                 qprobes_max=80):
        self.index = index
        h = ctypes.c_void_p()
        _check(lib().fpp_server_create(index.h, n_streams, memory_budget, max_batch, k_max, qprobes_max,
                                       ctypes.byref(h)))
        self.h = h
        self._keep = {}

    def submit(self, Q: np.ndarray, k: int, qprobes: int) -> int:
        Q = np.ascontiguousarray(Q, np.float32)
        out = np.zeros((Q.shape[0], k), np.int32)
        t = ctypes.c_longlong()
        _check(lib().fpp_server_submit(self.h, _ptr(Q), Q.shape[0], k, qprobes, _ptr(out), ctypes.byref(t)))
        self._keep[t.value] = (Q, out)
        return t.value

    def wait(self, ticket: int):
        lat = ctypes.c_double()
        _check(lib().fpp_server_wait(self.h, ticket, ctypes.byref(lat)))
        _, out = self._keep.pop(ticket)
        return out, lat.value

    def stats(self) -> dict:
        v = np.zeros(4, np.float64)
        _check(lib().fpp_server_stats(self.h, _ptr(v), 4))
        return dict(launches=int(v[0]), queries=int(v[1]), requests=int(v[2]), waiting=int(v[3]))

    def close(self):
        if self.h:
            lib().fpp_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def bruteforce_topk_f64(x_ptr: int, n: int, d: int, q_ptr: int, nq: int, k: int, out_ptr: int,
                        val_ptr: int | None = None, stream: int | None = None) -> None:
    """Exact FP64 MIPS top-k of device queries against device points (ground truth)."""
    _check(lib().fpp_bruteforce_topk_f64(ctypes.c_void_p(x_ptr), n, d, ctypes.c_void_p(q_ptr), nq, k,
                                         ctypes.c_void_p(out_ptr), ctypes.c_void_p(val_ptr or 0),
                                         ctypes.c_void_p(stream or 0)))


def load_txt(path: str, n_points: int, n_features: int):
    """The reference's loadtxtData (src/Utilities.cpp:42-61): n_points lines of
    n_features floats.  Returns (X, n_read): X is (n_points, n_features)
    float32, zero where the file runs short."""
    X = np.zeros((n_points, n_features), np.float32)
    got = ctypes.c_longlong(0)
    _check(lib().fpp_load_txt(os.fsencode(path), n_points, n_features, _ptr(X), ctypes.addressof(got)))
    return X, got.value


def output_file(path: str, topk: np.ndarray) -> None:
    """The reference's outputFile (src/Utilities.cpp:13-33): one query per line."""
    t = np.ascontiguousarray(topk, dtype=np.int32)
    _check(lib().fpp_output_file(os.fsencode(path), _ptr(t), t.shape[0], t.shape[1]))
