"""Load the reference chompack's pure-Python symbolic module under the cvxopt
shim (test infrastructure; only `make_golden.py` uses it, in a container where
the reference tree is present).

The reference package's `__init__` pulls in modules that need the real cvxopt
(solvers, conversion, ...), so a bare package object is registered instead and
only `chompack.misc` and `chompack.symbolic` are executed from the reference
sources (`src/python/misc.py`, `src/python/symbolic.py`).
"""
import os
import sys
import types

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.environ.get("CHOMPACK_REFERENCE", "/root/reference")


def load_reference():
    shim = os.path.join(HERE, "shim")
    if shim not in sys.path:
        sys.path.insert(0, shim)
    import cvxopt  # noqa: F401  (the shim)
    if "chompack.symbolic" in sys.modules:
        return sys.modules["chompack.symbolic"], sys.modules["chompack.misc"]
    pkg = types.ModuleType("chompack")
    pkg.__path__ = [os.path.join(REF, "src", "python")]
    sys.modules["chompack"] = pkg
    import importlib
    misc = importlib.import_module("chompack.misc")
    symbolic = importlib.import_module("chompack.symbolic")
    return symbolic, misc
