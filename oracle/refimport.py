"""Load the reference flexmm package (test infrastructure only).

The reference is pure Python + Numba.  It is not vendored: ``build_ref()``
copies its ``flexmm`` package from the read-only reference checkout into
``oracle/_ref/`` (git-ignored; the numba ``cache=True`` decorators in
flexmm/tree.py:10 need a writable directory).  ``load_reference()`` imports
that copy after applying the host shims the reference needs on this
Python/numpy:

* ``collections.MutableMapping`` (removed in Python 3.10; used by
  flexmm/flexmm2d/float_dict.py:1 and flexmm/kifmm2d/float_dict.py:1);
* ``np.Inf`` (removed in numpy 2; flexmm/kifmm2d/scalar/helpers.py:244);
* a numpy-backed ``numexpr.evaluate`` (numexpr is not installed;
  flexmm/kifmm2d/vector/stokes_fmm.py:3).

Only tests, golden-fixture generation and the reference arm of ``bench.py``
use this module.
"""
import collections
import collections.abc
import os
import shutil
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_COPY = os.path.join(HERE, "_ref")
# the read-only reference checkout; FLEXMM_REFERENCE overrides where it lies
REFERENCE_CHECKOUT = os.environ.get("FLEXMM_REFERENCE", "/root/reference")


def build_ref(src=REFERENCE_CHECKOUT, dst=REF_COPY):
    """Copy the reference package into ``oracle/_ref`` (no-op if absent)."""
    pkg = os.path.join(src, "flexmm")
    if not os.path.isdir(pkg):
        return False
    target = os.path.join(dst, "flexmm")
    if os.path.isdir(target):
        shutil.rmtree(target)
    os.makedirs(dst, exist_ok=True)
    shutil.copytree(pkg, target, ignore=shutil.ignore_patterns("__pycache__", "*.nbi", "*.nbc"))
    return True


def reference_available(dst=REF_COPY):
    return os.path.isfile(os.path.join(dst, "flexmm", "tree.py"))


def _apply_shims():
    collections.MutableMapping = collections.abc.MutableMapping
    if not hasattr(np, "Inf"):
        np.Inf = np.inf
    if "numexpr" not in sys.modules:
        try:
            import numexpr  # noqa: F401
        except ImportError:
            ne = types.ModuleType("numexpr")

            def evaluate(expr, out=None, local_dict=None):
                frame = sys._getframe(1)
                env = dict(frame.f_globals)
                env.update(frame.f_locals)
                if local_dict:
                    env.update(local_dict)
                env.setdefault("log", np.log)
                env.setdefault("exp", np.exp)
                env.setdefault("sqrt", np.sqrt)
                res = eval(expr, env)
                if out is not None:
                    out[...] = res
                    return out
                return res

            ne.evaluate = evaluate
            sys.modules["numexpr"] = ne


def load_reference(dst=REF_COPY):
    """Import and return the reference ``flexmm`` package from ``oracle/_ref``."""
    if not reference_available(dst):
        raise RuntimeError("reference copy missing: run oracle.refimport.build_ref() where the "
                           "reference checkout exists")
    _apply_shims()
    if dst not in sys.path:
        sys.path.insert(0, dst)
    import flexmm  # noqa: F401
    import flexmm.flexmm2d.kifmm  # noqa: F401
    import flexmm.flexmm2d.bbfmm  # noqa: F401
    return sys.modules["flexmm"]
