"""Saving and loading a built index: a fresh handle loaded from the file
holds the same sign bits, centre and bucket tables and answers every query
form with the same ids as the index that was saved; damaged or mismatched
files are rejected before the handle uses them."""
import numpy as np
import pytest

from falconnpp_b200 import capi, synth

pytestmark = pytest.mark.gpu


def _built(X, L=8, D=256, minSize=40, alpha=0.01, iProbes=3):
    g = capi.Index(*X.shape)
    g.set_index_param(L, D, minSize, alpha, iProbes, 8, 42)
    g.build(X)
    return g


def test_save_load_round_trip(tmp_path):
    X = synth.mixture(20000, 200, n_centres=32, seed=0)
    Q = synth.mixture(300, 200, n_centres=32, seed=1)
    g = _built(X)
    path = str(tmp_path / "index.fpp")
    g.save(path)
    h = capi.Index(*X.shape)
    h.load(path)
    b1, b2 = g.dump_bits()
    c1, c2 = h.dump_bits()
    assert np.array_equal(b1, c1) and np.array_equal(b2, c2)
    assert np.array_equal(g.dump_center().view(np.uint32), h.dump_center().view(np.uint32))
    s1, i1 = g.dump_tables()
    s2, i2 = h.dump_tables()
    assert np.array_equal(s1, s2) and np.array_equal(i1, i2)
    for qp in (5, 20):
        g.set_qprobes(qp)
        h.set_qprobes(qp)
        for form, prec in ((0, 0), (1, 0), (1, 2)):
            g.set_query_form(form, prec, 4)
            h.set_query_form(form, prec, 4)
            assert np.array_equal(g.query(Q, 10), h.query(Q, 10)), (qp, form, prec)
    g.close()
    h.close()


def test_load_rejects_bad_files(tmp_path):
    X = synth.mixture(3000, 64, n_centres=8, seed=0)
    g = _built(X, L=4, D=64, minSize=20, iProbes=2)
    path = tmp_path / "index.fpp"
    g.save(str(path))
    data = path.read_bytes()
    h = capi.Index(*X.shape)
    h.load(str(path))  # the good file first: a later rejected header leaves this index in place
    truncated = tmp_path / "truncated.fpp"
    truncated.write_bytes(data[:-4])
    with pytest.raises(capi.FppError):
        h.load(str(truncated))
    h.set_qprobes(4)
    h.query(synth.mixture(5, 64, n_centres=8, seed=1), 5)  # still built
    bad_magic = tmp_path / "magic.fpp"
    bad_magic.write_bytes(b"X" + data[1:])
    with pytest.raises(capi.FppError):
        h.load(str(bad_magic))
    # an id past n_points in the last section: rejected, the handle ends unbuilt
    bad_id = bytearray(data)
    bad_id[-4:] = np.array([3000], np.int32).tobytes()
    p = tmp_path / "bad_id.fpp"
    p.write_bytes(bytes(bad_id))
    with pytest.raises(capi.FppError):
        h.load(str(p))
    with pytest.raises(capi.FppError):
        h.query(synth.mixture(5, 64, n_centres=8, seed=1), 5)
    other = capi.Index(2999, 64)  # a handle of another size
    with pytest.raises(capi.FppError):
        other.load(str(path))
    for idx in (g, h, other):
        idx.close()


def test_pybind_save_load(tmp_path):
    from falconnpp_b200 import FalconnPP
    X = synth.mixture(5000, 100, n_centres=8, seed=0)
    Q = synth.mixture(50, 100, n_centres=8, seed=1)
    a = FalconnPP.FalconnPP(5000, 100)
    a.setIndexParam(n_tables=6, n_proj=128, bucket_minSize=20, bucket_scale=0.01, iProbes=2, random_seed=42)
    a.build(X.T)
    a.set_qProbes(8)
    ref = a.query(Q.T, 10)
    path = str(tmp_path / "a.fpp")
    a.save(path)
    b = FalconnPP.FalconnPP(5000, 100)
    b.load(path)
    b.set_qProbes(8)
    assert np.array_equal(b.query(Q.T, 10), ref)
