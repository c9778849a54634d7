"""The reference's text matrix formats (src/Utilities.cpp:13-61) through the
C ABI: loadtxtData reads n lines of d whitespace-separated floats (zeros
where the file runs short; a missing file is an error), outputFile writes one
query per line with a space after every id.  Host-only: no GPU needed."""
import numpy as np
import pytest

from falconnpp_b200 import capi


def test_loadtxt_round_trip_exact(tmp_path):
    rng = np.random.default_rng(0)
    X = (rng.standard_normal((37, 11)) * 10 ** rng.uniform(-3, 3, (37, 1))).astype(np.float32)
    p = tmp_path / "data.txt"
    with open(p, "w") as f:
        for row in X:
            f.write(" ".join("%.9g" % v for v in row) + "\n")
    got, n = capi.load_txt(str(p), 37, 11)
    assert n == 37 * 11
    assert np.array_equal(got.view(np.uint32), X.view(np.uint32))


def test_loadtxt_short_file_leaves_zeros(tmp_path):
    p = tmp_path / "short.txt"
    p.write_text("1 2 3\n4 5\n")
    got, n = capi.load_txt(str(p), 3, 3)
    assert n == 5
    assert np.array_equal(got, np.array([[1, 2, 3], [4, 5, 0], [0, 0, 0]], np.float32))


def test_loadtxt_missing_file_is_an_error(tmp_path):
    with pytest.raises(capi.FppError) as e:
        capi.load_txt(str(tmp_path / "nope.txt"), 2, 2)
    assert e.value.code == capi.FPP_ERR_INVALID_ARGUMENT


def test_output_file_format(tmp_path):
    topk = np.array([[5, 3, 0], [12, 7, 1]], np.int32)
    p = tmp_path / "out.txt"
    capi.output_file(str(p), topk)
    assert p.read_text() == "5 3 0 \n12 7 1 \n"


def test_pybind_text_functions(tmp_path):
    from falconnpp_b200 import FalconnPP
    p = tmp_path / "d.txt"
    p.write_text("1 2\n3 4\n5 6\n")
    X = FalconnPP.loadtxtData(str(p), 3, 2)
    assert X.shape == (2, 3) and X.flags["F_CONTIGUOUS"]
    assert np.array_equal(X, np.array([[1, 3, 5], [2, 4, 6]], np.float32))
    o = tmp_path / "o.txt"
    FalconnPP.outputFile(np.array([[9, 8]], np.int32), str(o))
    assert o.read_text() == "9 8 \n"
