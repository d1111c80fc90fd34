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
        dd = _lib.oracle_direct_laplace_dipole
        dd.argtypes = [dp, dp, dp, dp, dp, dp, ctypes.c_int64, dp, dp, ctypes.c_int64, ctypes.c_int, dp]
        dd.restype = None
        sd = _lib.oracle_direct_stokes_dipole
        sd.argtypes = [dp] * 8 + [ctypes.c_int64, dp, dp, ctypes.c_int64, ctypes.c_int, dp]
        sd.restype = None
        h = _lib.oracle_direct_stokes
        h.argtypes = [dp, dp, dp, dp, ctypes.c_int64, dp, dp, ctypes.c_int64, ctypes.c_int, dp]
        h.restype = None
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


def direct_laplace_dipole(sx, sy, slp, dlp, nx, ny, tx, ty, check):
    """FP64 direct sum of the Laplace single + double layer
    (examples/pure_kifmm_laplace_dipoles.py:31-40)."""
    lib = _load()
    a = [np.ascontiguousarray(v, dtype=np.float64) for v in (sx, sy, slp, dlp, nx, ny, tx, ty)]
    out = np.empty(a[6].size)
    lib.oracle_direct_laplace_dipole(*[_p(v) for v in a[:6]], a[0].size, _p(a[6]), _p(a[7]),
                                     a[6].size, 1 if check else 0, _p(out))
    return out


def direct_laplace_grad(sx, sy, tau, tx, ty, check):
    """FP64 direct sum of the Laplace potential and its target gradient -> [3, nt]."""
    lib = _load()
    sx, sy, tau, tx, ty = (np.ascontiguousarray(a, dtype=np.float64) for a in (sx, sy, tau, tx, ty))
    out = np.empty((3, tx.size))
    lib.oracle_direct_laplace_grad(_p(sx), _p(sy), _p(tau), sx.size, _p(tx), _p(ty), tx.size,
                                   1 if check else 0, _p(out))
    return out


def _mh_pairs(sx, sy, tau, tx, ty, k, check, grad):
    """Chunked numpy/scipy direct sum of K0(k r)/(2 pi) (and its target gradient)."""
    from scipy.special import k0, k1
    nt = tx.size
    out = np.zeros((3 if grad else 1, nt))
    step = max(1, 4_000_000 // max(sx.size, 1))
    for a in range(0, nt, step):
        b = min(nt, a + step)
        dx = tx[a:b, None] - sx[None, :]
        dy = ty[a:b, None] - sy[None, :]
        r = np.sqrt(dx * dx + dy * dy)
        skip = (dx == 0) & (dy == 0) if check else np.zeros(r.shape, dtype=bool)
        rs = np.where(skip, 1.0, r)
        w = np.where(skip, 0.0, tau[None, :])
        out[0, a:b] = (k0(k * rs) / (2 * np.pi) * w).sum(1)
        if grad:
            s = -k * k1(k * rs) / rs / (2 * np.pi) * w
            out[1, a:b] = (s * dx).sum(1)
            out[2, a:b] = (s * dy).sum(1)
    return out


def direct_mod_helmholtz(sx, sy, tau, tx, ty, k, check):
    """FP64 direct sum of the modified Helmholtz kernel K0(k r)/(2 pi)
    (examples/kifmm_modified_helmholtz.py:33-39), skipping coincident pairs
    when ``check``; K0 from scipy.special (test infrastructure only)."""
    a = [np.ascontiguousarray(v, dtype=np.float64) for v in (sx, sy, tau, tx, ty)]
    return _mh_pairs(*a, float(k), check, False)[0]


def direct_mod_helmholtz_grad(sx, sy, tau, tx, ty, k, check):
    """Potential and target gradient of the modified Helmholtz kernel -> [3, nt]
    (examples/pure_kifmm_modified_helmholtz_gradient.py:45-70)."""
    a = [np.ascontiguousarray(v, dtype=np.float64) for v in (sx, sy, tau, tx, ty)]
    return _mh_pairs(*a, float(k), check, True)


def struve_gf(x):
    """The Struve Green's function of examples/bbfmm_struve.py:29-33, scipy.

    scipy's struve returns NaN on short intervals (measured: order -2 near
    x = 25.8463 and 28.995, order -3 near 27.329, each ~3e-5 wide); there the
    value is the cubic through GF at x +- 1e-4 and x +- 2e-4, outside them
    (GF is smooth on that scale: interpolation error ~1e-15 relative)."""
    from scipy.special import struve, yn

    def gf(v):
        return (v * (yn(1, v) - struve(-3, v)) - 4 * struve(-2, v)) / v ** 2
    x = np.asarray(x, dtype=np.float64)
    out = gf(x)
    bad = ~np.isfinite(out)
    if np.any(bad):
        xb = x[bad]
        h = 1e-4
        f = [gf(xb + k * h) for k in (-2, -1, 1, 2)]
        # Lagrange weights of the nodes -2h, -h, h, 2h at 0
        out[bad] = (-f[0] + 4 * f[1] + 4 * f[2] - f[3]) / 6.0
    return out


def direct_radial(f, sx, sy, tau, tx, ty, check):
    """FP64 direct sum of a radial kernel f(|t - s|) (numpy; test infrastructure)."""
    sx, sy, tau, tx, ty = (np.ascontiguousarray(v, dtype=np.float64) for v in (sx, sy, tau, tx, ty))
    out = np.zeros(tx.size)
    step = max(1, 2_000_000 // max(sx.size, 1))
    for a in range(0, tx.size, step):
        b = min(tx.size, a + step)
        dx = tx[a:b, None] - sx[None, :]
        dy = ty[a:b, None] - sy[None, :]
        r = np.sqrt(dx * dx + dy * dy)
        skip = (dx == 0) & (dy == 0) if check else np.zeros(r.shape, dtype=bool)
        out[a:b] = (f(np.where(skip, 1.0, r)) * np.where(skip, 0.0, tau[None, :])).sum(1)
    return out


def direct_stokes(sx, sy, fx, fy, tx, ty, check):
    """FP64 Stokeslet direct sum -> [3, nt] rows (u, v, p)."""
    lib = _load()
    sx, sy, fx, fy, tx, ty = (np.ascontiguousarray(a, dtype=np.float64) for a in (sx, sy, fx, fy, tx, ty))
    out = np.empty((3, tx.size))
    lib.oracle_direct_stokes(_p(sx), _p(sy), _p(fx), _p(fy), sx.size, _p(tx), _p(ty), tx.size,
                             1 if check else 0, _p(out))
    return out


def direct_stokes_dipole(sx, sy, fx, fy, gx, gy, nx, ny, tx, ty, check):
    """FP64 direct sum of Stokeslets plus stresslets -> [3, nt] rows (u, v, p)
    (flexmm/kifmm2d/vector/stokes_fmm.py:128-235)."""
    lib = _load()
    a = [np.ascontiguousarray(v, dtype=np.float64) for v in (sx, sy, fx, fy, gx, gy, nx, ny, tx, ty)]
    out = np.empty((3, a[8].size))
    lib.oracle_direct_stokes_dipole(*[_p(v) for v in a[:8]], a[0].size, _p(a[8]), _p(a[9]),
                                    a[8].size, 1 if check else 0, _p(out))
    return out
