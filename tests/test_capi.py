"""The C-ABI library loads, exports every function include/falconnpp_b200.h
declares, and the pybind module mirrors the reference's Python surface
(python/python_wrapper.cpp:14-30).  No compute runs here (no GPU needed)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    src = open(os.path.join(ROOT, "include", "falconnpp_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(fpp_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    from falconnpp_b200 import LIBRARY_PATH, capi
    lib = ctypes.CDLL(LIBRARY_PATH)
    declared = header_functions()
    assert len(declared) >= 20
    missing = [f for f in declared if not hasattr(lib, f)]
    assert not missing, missing
    assert sorted(capi.EXPORTED) == declared


def test_library_is_built_for_sm100a_only():
    # the flags the build recorded when it compiled and linked the library:
    # every -gencode names sm_100a and nothing else, no fast-math, no FMA
    # contraction (the bit-exact FP32 path depends on it)
    import json
    from falconnpp_b200 import _build
    with open(_build.FLAGS_FILE) as f:
        rec = json.load(f)
    for flags in (rec["compile"], rec["link"]):
        gencodes = [flags[i + 1] for i, x in enumerate(flags) if x == "-gencode"]
        assert gencodes == ["arch=compute_100a,code=sm_100a"], gencodes
    assert "-fmad=false" in rec["compile"] and "-ftz=false" in rec["compile"]
    assert not any("fast-math" in x for x in rec["compile"])
    assert sorted(rec["sources"]) == sorted(_build.CU_SOURCES)


def test_pybind_module_mirrors_reference_api():
    from falconnpp_b200 import FalconnPP
    cls = FalconnPP.FalconnPP
    for name in ["setIndexParam", "set_qProbes", "set_threads", "clear", "build", "query", "build2D", "query2D"]:
        assert hasattr(cls, name), name
    doc = cls.setIndexParam.__doc__
    for kw in ["n_tables", "n_proj", "bucket_minSize", "bucket_scale", "iProbes"]:
        assert kw in doc, (kw, doc)
    assert re.search(r"n_threads: [^,]*= 8", doc) and re.search(r"random_seed: [^)]*= -1", doc)
    assert "n_neighbors" in cls.query.__doc__ and "verbose: bool = False" in cls.query.__doc__


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks the no-GPU error path")
def test_fails_loudly_without_gpu():
    from falconnpp_b200 import FalconnPP, capi
    with pytest.raises(capi.FppError) as e:
        capi.Index(100, 8)
    assert e.value.code == -7
    with pytest.raises(RuntimeError):
        FalconnPP.FalconnPP(100, 8)


def test_oracle_is_not_linked_by_the_product():
    import subprocess
    from falconnpp_b200 import LIBRARY_PATH
    deps = subprocess.run(["ldd", LIBRARY_PATH], capture_output=True, text=True).stdout
    assert "oracle" not in deps
    for root, _, files in os.walk(os.path.join(ROOT, "falconnpp_b200")):
        for f in files:
            if f.endswith((".py", ".cu", ".cuh", ".h", ".cpp")):
                txt = open(os.path.join(root, f)).read()
                assert "import oracle" not in txt and "from oracle" not in txt, f
