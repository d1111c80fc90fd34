"""ctypes front end of oracle/direct.c (test infrastructure only)."""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "direct.c")
LIB = os.path.join(HERE, "_build", "liboracle_direct.so")
_lib = None


def build():
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(SRC):
        subprocess.check_call(["gcc", "-O2", "-fopenmp", "-shared", "-fPIC", SRC, "-o", LIB, "-lm"])
    return LIB


def _load():
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(build())
        dp = ctypes.POINTER(ctypes.c_double)
        f = _lib.oracle_direct_laplace
        f.argtypes = [dp, dp, dp, ctypes.c_int64, dp, dp, ctypes.c_int64, ctypes.c_int, dp]
        f.restype = None
        g = _lib.oracle_direct_laplace_grad
        g.argtypes = f.argtypes
        g.restype = None
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def direct_laplace(sx, sy, tau, tx, ty, check):
    lib = _load()
    sx, sy, tau, tx, ty = (np.ascontiguousarray(a, dtype=np.float64) for a in (sx, sy, tau, tx, ty))
    out = np.empty(tx.size)
    lib.oracle_direct_laplace(_p(sx), _p(sy), _p(tau), sx.size, _p(tx), _p(ty), tx.size,
                              1 if check else 0, _p(out))
    return out


def direct_laplace_grad(sx, sy, tau, tx, ty, check):
    """FP64 direct sum of the Laplace potential and its target gradient -> [3, nt]."""
    lib = _load()
    sx, sy, tau, tx, ty = (np.ascontiguousarray(a, dtype=np.float64) for a in (sx, sy, tau, tx, ty))
    out = np.empty((3, tx.size))
    lib.oracle_direct_laplace_grad(_p(sx), _p(sy), _p(tau), sx.size, _p(tx), _p(ty), tx.size,
                                   1 if check else 0, _p(out))
    return out
