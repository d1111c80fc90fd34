"""Kernel registry: the reference's example kernels as device functors.

The reference takes a numba ``@njit`` scalar function ``K(sx, sy, tx, ty)``
and inlines it into every loop (flexmm/flexmm2d/helpers.py:87-151).  Here a
kernel is a ``Kernel`` naming a CUDA device functor compiled into
``libflexmm_b200.so``, plus a vectorised numpy twin used only to form the
per-width translation operators on the host (the reference forms them with
the same scalar function, flexmm/flexmm2d/kifmm.py:18-62).

A user's own numba function is accepted when its ``__name__`` is a
registered name, so scripts written for the reference work unchanged::

    @numba.njit(fastmath=True)
    def Laplace_Eval(sx, sy, tx, ty): ...
    KI_FMM(px, py, Laplace_Eval, Ncutoff, Nequiv)
"""
import numpy as np


class Kernel:
    vector = False   # vector-valued kernels (Stokes) have their own FMM class

    def __init__(self, name, kernel_id, params, host):
        self.name = name
        self.kernel_id = kernel_id
        self.params = tuple(float(p) for p in params) + (0.0,) * (4 - len(params))
        self._host = host

    def host(self, sx, sy, tx, ty):
        """Vectorised FP64 evaluation on the host (operator formation only)."""
        return self._host(self.params, sx, sy, tx, ty)

    @property
    def key(self):
        return (self.name, self.params)

    def __repr__(self):
        return f"Kernel({self.name}, params={self.params[:1]})"


def _laplace_host(p, sx, sy, tx, ty):
    # examples/kifmm_laplace.py:24-29
    dx = tx - sx
    dy = ty - sy
    d2 = dx * dx + dy * dy
    return -np.log(d2) / (4 * np.pi)


def _mod_helmholtz_host(p, sx, sy, tx, ty):
    # examples/kifmm_modified_helmholtz.py:33-39: K0(k d) / (2 pi)
    from scipy.special import k0
    dx = tx - sx
    dy = ty - sy
    return k0(p[0] * np.sqrt(dx * dx + dy * dy)) / (2 * np.pi)


KERNEL_LAPLACE = 0
KERNEL_MOD_HELMHOLTZ = 1
KERNEL_RADIAL_TABLE = 2


def _cheb_nodes(n):
    return np.cos(np.pi * (np.arange(n) + 0.5) / n)


def _clenshaw(c, u):
    b1 = np.zeros_like(u)
    b2 = np.zeros_like(u)
    for ci in c[:0:-1]:
        b1, b2 = 2 * u * b1 - b2 + ci, b1
    return u * b1 - b2 + c[0]


class RadialTable:
    """f(r) as Chebyshev series of degree n-1 on the octaves [2^j, 2^(j+1))
    covering [a, b] (the device evaluates the same table, csrc/kernels.cuh
    RadialTableF64).  The reference's examples tabulate their special-function
    kernels the same way with function_generator (FunctionGenerator(f, a, b,
    tol), examples/bbfmm_struve.py:34-36); octaves resolve a power-law or log
    singularity at 0 with a fixed degree."""

    def __init__(self, f, a, b, tol=1e-12, n=24):
        if not 0 < a < b:
            raise ValueError("need 0 < a < b")
        self.j0 = int(np.floor(np.log2(a)))
        j1 = int(np.ceil(np.log2(b)))
        self.noct = max(1, j1 - self.j0)
        self.n = int(n)
        u = _cheb_nodes(self.n)
        coef = np.empty((self.noct, self.n))
        k = np.arange(self.n)
        cosm = np.cos(np.pi * np.outer(np.arange(self.n), k + 0.5) / self.n)
        rng = np.random.default_rng(0)
        worst = 0.0
        for o in range(self.noct):
            lo = 2.0 ** (self.j0 + o)
            fx = np.asarray(f(lo * (1.5 + 0.5 * u)), dtype=np.float64)
            if not np.all(np.isfinite(fx)):
                raise ValueError(f"f is not finite on [{lo}, {2 * lo})")
            c = 2.0 / self.n * cosm.dot(fx)
            c[0] *= 0.5
            coef[o] = c
            uc = rng.uniform(-1, 1, 3 * self.n)
            ref = np.asarray(f(lo * (1.5 + 0.5 * uc)), dtype=np.float64)
            err = np.abs(_clenshaw(c, uc) - ref) / np.maximum(np.abs(ref), 1e-300)
            worst = max(worst, float(err.max()))
        if worst > tol:
            raise ValueError(f"tabulation error {worst:.1e} above tol {tol:.1e}; raise n")
        self.coef = np.ascontiguousarray(coef)
        self.max_rel_err = worst
        self.table_id = None

    def __call__(self, r):
        """Host evaluation of the tabulated f (operator formation)."""
        r = np.asarray(r, dtype=np.float64)
        lo, hi = 2.0 ** self.j0, 2.0 ** (self.j0 + self.noct)
        r = np.clip(r, lo, hi * (1 - 1e-16))
        _, e = np.frexp(r)
        o = e - 1 - self.j0
        a = np.ldexp(1.0, e - 1)
        u = (2 * r - 3 * a) / a
        c = self.coef[o]
        b1 = np.zeros_like(u)
        b2 = np.zeros_like(u)
        for i in range(self.n - 1, 0, -1):
            b1, b2 = 2 * u * b1 - b2 + c[..., i], b1
        return u * b1 - b2 + c[..., 0]

    def register(self):
        """Upload to the library (once); returns the table id."""
        if self.table_id is None:
            import ctypes
            from . import _lib
            tid = ctypes.c_int(-1)
            _lib.call("fmm_kernel_table_create", self.coef.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                      self.j0, self.noct, self.n, ctypes.byref(tid))
            self.table_id = tid.value
        return self.table_id


def radial(f, a, b, tol=1e-12, n=24, name="Radial"):
    """A kernel K(s, t) = f(|t - s|) from any vectorised function f, tabulated
    on [a, b] (the reference's ``FunctionGenerator(f, a, b, tol)`` plus the
    scalar kernel that calls it, e.g. examples/bbfmm_struve.py:29-46)."""
    table = RadialTable(f, a, b, tol=tol, n=n)
    tid = table.register()

    def host(p, sx, sy, tx, ty):
        dx = tx - sx
        dy = ty - sy
        return table(np.sqrt(dx * dx + dy * dy))
    k = Kernel(name, KERNEL_RADIAL_TABLE, (tid, table.j0, table.noct, table.n), host)
    k.table = table
    return k


def Laplace():
    return Kernel("Laplace_Eval", KERNEL_LAPLACE, (), _laplace_host)


def ModifiedHelmholtz(helmholtz_k):
    """K0(k |t - s|) / (2 pi), k = helmholtz_k > 0."""
    if not helmholtz_k > 0:
        raise ValueError("helmholtz_k must be positive")
    return Kernel("Modified_Helmholtz_Eval", KERNEL_MOD_HELMHOLTZ, (helmholtz_k,),
                  _mod_helmholtz_host)


def struve_gf(x):
    """The Struve Green's function GF(r) = (r (Y1(r) - H_-3(r)) - 4 H_-2(r)) / r^2
    of examples/bbfmm_struve.py:29-33, from scipy's Bessel and Struve
    functions.  scipy's struve returns NaN on a few ~3e-5-wide intervals
    (order -2 near r = 25.8463 and 28.995, order -3 near 27.329); there GF is
    taken from the cubic through its values at r +- 1e-4 and r +- 2e-4."""
    from scipy.special import struve, yn

    def gf(v):
        return (v * (yn(1, v) - struve(-3, v)) - 4 * struve(-2, v)) / v ** 2
    x = np.asarray(x, dtype=np.float64)
    out = np.asarray(gf(x), dtype=np.float64)
    bad = ~np.isfinite(out)
    if np.any(bad):
        xb = x[bad]
        h = 1e-4
        f = [gf(xb + k * h) for k in (-2, -1, 1, 2)]
        out[bad] = (-f[0] + 4 * f[1] + 4 * f[2] - f[3]) / 6.0
    return out


_STRUVE = {}


def Struve(b=256.0):
    """The Struve example's kernel ``Kernel`` (examples/bbfmm_struve.py:29-46):
    GF(|t - s|) tabulated on [1e-30, b] as the example tabulates it with
    function_generator (there b = 1000; here 256 by default: beyond it scipy's
    GF loses most of its relative digits to cancellation, |GF| < 1e-11 there,
    and distances above b are clamped to b).  One table per process and b."""
    b = float(b)
    if b not in _STRUVE:
        _STRUVE[b] = radial(struve_gf, 1e-30, b, tol=1e-5, name="Kernel")
    return _STRUVE[b]


KERNEL_STOKES = 3


def _stokes_host(p, sx, sy, tx, ty):
    """The Stokeslet (u, v, p) rows for unit forces in x and y
    (kifmm2d/vector/stokes_fmm.py:161-184): [3, 2, ...] = rows (u, v, p) by
    force component (fx, fy)."""
    dx = tx - sx
    dy = ty - sy
    d2 = dx * dx + dy * dy
    il = 1.0 / d2
    lg = -0.5 * np.log(d2)
    f4 = 1.0 / (4 * np.pi)
    f2 = 1.0 / (2 * np.pi)
    return np.array([[f4 * (lg + dx * dx * il), f4 * dx * dy * il],
                     [f4 * dx * dy * il, f4 * (lg + dy * dy * il)],
                     [f2 * dx * il, f2 * dy * il]])


def Stokes():
    """The 2D Stokeslet of the reference's Stokes FMM (vector valued: forces
    (fx, fy) in, (u, v, p) out; kifmm2d/vector/stokes_fmm.py:100-187).  Its
    FMM is ``flexmm_b200.stokes.FMM``, as in the reference; the scalar FMM
    classes refuse it."""
    k = Kernel("Stokes", KERNEL_STOKES, (), _stokes_host)
    k.vector = True
    return k


_BY_NAME = {"Laplace_Eval": Laplace, "Laplace": Laplace,
            "Modified_Helmholtz_Eval": ModifiedHelmholtz, "ModifiedHelmholtz": ModifiedHelmholtz,
            "Kernel": Struve, "Struve": Struve,
            "Stokes": Stokes, "Stokes_Kernel_Form": Stokes}
# parameters a reference-style kernel function reads from its module's globals
_GLOBAL_PARAMS = {"Modified_Helmholtz_Eval": ("helmholtz_k",)}


def _function_globals(fn):
    fn = getattr(fn, "py_func", fn)  # numba dispatcher -> python function
    return getattr(fn, "__globals__", {})


def resolve(kernel_eval, **params):
    """Map a Kernel, a registered name, or a function named like one to a Kernel.

    The reference's example kernels close over module globals (the modified
    Helmholtz example reads ``helmholtz_k``); a function passed here supplies
    such a parameter the same way unless it is given as a keyword."""
    if isinstance(kernel_eval, Kernel):
        return kernel_eval
    name = kernel_eval if isinstance(kernel_eval, str) else getattr(kernel_eval, "__name__", None)
    if name not in _BY_NAME:
        raise ValueError(f"kernel {name!r} is not registered; registered: {sorted(_BY_NAME)}")
    for key in _GLOBAL_PARAMS.get(name, ()):
        if key not in params:
            g = _function_globals(kernel_eval) if not isinstance(kernel_eval, str) else {}
            if key not in g:
                raise ValueError(f"kernel {name!r} needs {key}= (or a module global {key})")
            params[key] = float(g[key])
    return _BY_NAME[name](**params)
