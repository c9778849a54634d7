"""B200-native Falconn++ (locality-sensitive filtering for maximum inner
product search) behind the reference's API.

* ``falconnpp_b200.FalconnPP`` is the pybind11 module with the reference's
  class ``FalconnPP`` (``setIndexParam``, ``build``, ``set_qProbes``,
  ``query``, ...); ``from falconnpp_b200 import FalconnPP`` followed by
  ``FalconnPP.FalconnPP(n, d)`` reads like the reference's
  ``import FalconnPP``.
* ``falconnpp_b200.capi`` is a thin ctypes view of the C ABI
  (include/falconnpp_b200.h), used by the tests and the benchmark.

Both fail loudly if the native library has not been built
(``python -m falconnpp_b200._build``): there is no CPU fallback.
"""
import os as _os

_HERE = _os.path.dirname(_os.path.abspath(__file__))
LIBRARY_PATH = _os.path.join(_HERE, "libfalconnpp_b200.so")


def _require_native():
    if not _os.path.exists(LIBRARY_PATH):
        raise ImportError(
            "falconnpp_b200: native library missing at %s; build it with "
            "`python -m falconnpp_b200._build`" % LIBRARY_PATH)


def __getattr__(name):
    if name == "FalconnPP":
        _require_native()
        import importlib
        mod = importlib.import_module(".FalconnPP", __name__)
        globals()["FalconnPP"] = mod
        return mod
    raise AttributeError(name)
