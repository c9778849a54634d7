"""Error paths of the boundary.  The reference leaves these undefined
(src/FalconnPP.h:85-100 validates nothing); the C ABI rejects them with a
status code and a message, and pybind maps the codes to ValueError /
RuntimeError.  Allocation failures are injected on the host
("inject_alloc_failure": the n-th device allocation from then on fails once,
without calling cudaMalloc), so no test faults the GPU: every allocation of a
build, a plain query and a batched query is failed in turn, each failure
must come back as FPP_ERR_OUT_OF_MEMORY, and the handle must stay usable and
give the clean result afterwards."""
import numpy as np
import pytest

from falconnpp_b200 import capi, synth

pytestmark = pytest.mark.gpu

INVALID, NOT_BUILT, OOM, UNSUPPORTED, NON_FINITE = -1, -2, -4, -5, -6


def _code(fn, *a):
    with pytest.raises(capi.FppError) as e:
        fn(*a)
    return e.value.code


def test_index_param_rejections():
    g = capi.Index(1000, 20)
    assert _code(g.set_index_param, 4, 100, 10, 0.1, 1) == INVALID   # n_proj not a power of two
    assert _code(g.set_index_param, 4, 0, 10, 0.1, 1) == INVALID
    assert _code(g.set_index_param, 4, 16, 10, 0.1, 0) == INVALID    # iProbes < 1
    assert _code(g.set_index_param, 4, 8, 10, 0.1, 16) == INVALID    # iProbes > n_proj
    assert _code(g.set_index_param, 4, 64, 10, 0.1, 33) == INVALID   # iProbes > 32
    assert _code(g.set_index_param, 4, 16, 10, float("nan"), 1) == INVALID
    assert _code(g.set_index_param, 4, 16, 10, -1.0, 1) == INVALID
    assert _code(g.set_index_param, 0, 16, 10, 0.1, 1) == INVALID    # n_tables < 1
    assert _code(g.set_index_param, 4, 2048, 10, 0.1, 1) == UNSUPPORTED  # fhtDim > 1024
    g.set_index_param(4, 16, 10, 0.1, 1, 8, 1)  # a valid call still works afterwards
    g.close()


def test_call_order_and_query_rejections():
    X = synth.mixture(2000, 16, n_centres=4, seed=0)
    Q = synth.mixture(8, 16, n_centres=4, seed=1)
    g = capi.Index(*X.shape)
    assert _code(g.build, X) == INVALID                     # setIndexParam first
    g.set_index_param(1, 4, 10, 0.1, 1, 8, 1)
    assert _code(g.query, Q, 5) == NOT_BUILT
    g.build(X)
    g.set_qprobes(8)                                         # m = 16, m1 = 4 = n_proj: allowed
    assert g.query(Q, 5).shape == (8, 5)
    g.set_qprobes(9)                                         # m = 18, m1 = 5 > n_proj = 4
    assert _code(g.query, Q, 5) == INVALID
    assert b"qProbes too large" in capi.lib().fpp_last_error()
    g.set_qprobes(2)
    assert _code(g.query, Q, 0) == INVALID                   # n_neighbors < 1
    assert _code(g.query, Q, 1025) == INVALID                # n_neighbors > 1024
    assert _code(g.set_qprobes, 0) == INVALID
    g.close()


@pytest.mark.parametrize("bad", [np.nan, np.inf, -np.inf])
def test_non_finite_data_rejected(bad):
    X = synth.mixture(1000, 16, n_centres=4, seed=0)
    X[123, 7] = bad
    g = capi.Index(*X.shape)
    g.set_index_param(2, 16, 10, 0.1, 1, 8, 1)
    assert _code(g.build, X) == NON_FINITE
    X[123, 7] = 0.0
    g.build(X)  # the same handle builds once the data is finite
    g.close()


def test_pybind_maps_codes_to_exceptions():
    from falconnpp_b200 import FalconnPP
    X = synth.mixture(1000, 16, n_centres=4, seed=0)
    idx = FalconnPP.FalconnPP(1000, 16)
    with pytest.raises(ValueError):
        idx.setIndexParam(2, 12, 10, 0.1, 1)
    with pytest.raises(ValueError):
        idx.build(np.transpose(X)[:, :10])  # wrong shape
    idx.setIndexParam(2, 16, 10, 0.1, 1)
    with pytest.raises(RuntimeError):
        idx.query(np.transpose(X[:4]), 5)   # not built


def _fail_each_allocation(g, reset, action, clean):
    """For n = 1, 2, ...: reset the handle, fail the n-th allocation of
    action(), and stop once action() completes without reaching it.  Every
    failure must be an out-of-memory status, after which the same handle,
    called again, gives the clean result."""
    failures = 0
    for nth in range(1, 200):
        reset()
        g.set_option("inject_alloc_failure", nth)
        try:
            got = action()
        except capi.FppError as e:
            assert e.code == OOM, (nth, e)
            failures += 1
            assert np.array_equal(action(), clean), f"handle unusable after failing allocation {nth}"
            continue
        g.set_option("inject_alloc_failure", 0)
        assert np.array_equal(got, clean)
        return failures
    raise AssertionError("the action never completed")


def test_injected_allocation_failures_leave_the_handle_usable():
    X = synth.mixture(6000, 40, n_centres=8, seed=0)
    Q = synth.mixture(50, 40, n_centres=8, seed=1)
    ref = capi.Index(*X.shape)
    ref.set_index_param(4, 64, 20, 0.05, 2, 8, 3)
    ref.build(X)
    ref.set_qprobes(6)
    clean = ref.query(Q, 10)
    ref.set_query_form(1, 2, 4)
    clean_fp8 = ref.query(Q, 10)
    g = capi.Index(*X.shape)
    g.set_index_param(4, 64, 20, 0.05, 2, 8, 3)
    g.set_qprobes(6)

    def rebuild():
        g.clear()
        g.build(X)

    def build_then_query():
        g.build(X)
        return g.query(Q, 10)

    try:
        # every allocation of a build and of the first plain query after it
        assert _fail_each_allocation(g, lambda: None, build_then_query, clean) >= 5
        # the plain query's workspace alone (clear() releases it)
        assert _fail_each_allocation(g, rebuild, lambda: g.query(Q, 10), clean) >= 1
        # the batched form: staging buffers, low-precision rows, per-block scratch
        g.set_query_form(1, 2, 4)
        assert _fail_each_allocation(g, rebuild, lambda: g.query(Q, 10), clean_fp8) >= 3
        g.set_query_form(0, 0, 4)
        assert np.array_equal(g.query(Q, 10), clean)
    finally:
        g.set_option("inject_alloc_failure", 0)
    g.close()
    ref.close()
