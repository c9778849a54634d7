"""Compile the native parts of falconnpp_b200 in-tree.

* ``libfalconnpp_b200.so``: the CUDA kernels and the C ABI
  (include/falconnpp_b200.h), built with nvcc for sm_100a only, no fast-math,
  no FMA contraction (``-fmad=false``: every float operation rounds as written,
  which the bit-exact FP32 path depends on);
* ``FalconnPP<ext>``: the pybind11 module with the reference's class API,
  linked against the library above (rpath $ORIGIN).

Run ``python -m falconnpp_b200._build`` or call :func:`build`.
"""
from __future__ import annotations

import os
import subprocess
import sys
import sysconfig
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libfalconnpp_b200.so")
CU_SOURCES = ["fpp_build.cu", "fpp_query.cu", "fpp_capi.cu", "fpp_batch.cu", "fpp_batch_f32.cu", "fpp_batch_bf16.cu",
              "fpp_batch_fp8.cu", "fpp_batch_big.cu", "fpp_batch_ext.cu", "fpp_noalloc.cu", "fpp_server.cu", "fpp_bruteforce.cu", "fpp_bf_lowp.cu", "fpp_persist.cu",
              "fpp_hash_verify.cu"]
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17", "-fmad=false", "-ftz=false", "-prec-div=true", "-prec-sqrt=true",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
]


def _nvcc() -> str:
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("command failed: " + " ".join(cmd) + "\n" + r.stdout + r.stderr)


def _newer(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(d) <= t for d in deps)


FLAGS_FILE = os.path.join(HERE, "_build", "build_flags.json")
LINK_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-shared"]


def _record_flags() -> None:
    """The flags the library's objects and link were made with (read by the
    tests to check the target architecture without inspecting the binary)."""
    import json
    with open(FLAGS_FILE, "w") as f:
        json.dump({"compile": NVCC_FLAGS, "link": LINK_FLAGS, "sources": CU_SOURCES}, f, indent=1)


def build_library(force: bool = False) -> str:
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(ROOT, "include", "falconnpp_b200.h"))
    sources = [s for s in CU_SOURCES if os.path.exists(os.path.join(CSRC, s))]
    objs = []
    jobs = []
    for s in sources:
        src = os.path.join(CSRC, s)
        obj = os.path.join(objdir, s.replace(".cu", ".o"))
        objs.append(obj)
        if force or not _newer(obj, [src] + headers):
            jobs.append([_nvcc(), *NVCC_FLAGS, "-c", src, "-o", obj])
    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        list(ex.map(_run, jobs))
    if force or jobs or not _newer(LIB, objs):
        _run([_nvcc(), *LINK_FLAGS, "-o", LIB, *objs, "-Xlinker", "--no-undefined"])
        _record_flags()
    elif not os.path.exists(FLAGS_FILE):
        _record_flags()
    return LIB


def build_module(force: bool = False) -> str:
    import pybind11

    ext = sysconfig.get_config_var("EXT_SUFFIX") or ".so"
    target = os.path.join(HERE, "FalconnPP" + ext)
    src = os.path.join(CSRC, "python_module.cpp")
    deps = [src, LIB, os.path.join(ROOT, "include", "falconnpp_b200.h")]
    if not force and _newer(target, deps):
        return target
    inc = [pybind11.get_include(), sysconfig.get_paths()["include"]]
    cmd = ["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-fvisibility=hidden",
           *[f"-I{i}" for i in inc], src, "-o", target,
           f"-L{HERE}", "-lfalconnpp_b200", "-Wl,-rpath,$ORIGIN"]
    _run(cmd)
    return target


def build(force: bool = False) -> None:
    build_library(force)
    build_module(force)


if __name__ == "__main__":
    build(force="--force" in sys.argv)
    print("built", LIB)
