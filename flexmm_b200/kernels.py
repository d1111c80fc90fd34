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


def Laplace():
    return Kernel("Laplace_Eval", KERNEL_LAPLACE, (), _laplace_host)


def ModifiedHelmholtz(helmholtz_k):
    """K0(k |t - s|) / (2 pi), k = helmholtz_k > 0."""
    if not helmholtz_k > 0:
        raise ValueError("helmholtz_k must be positive")
    return Kernel("Modified_Helmholtz_Eval", KERNEL_MOD_HELMHOLTZ, (helmholtz_k,),
                  _mod_helmholtz_host)


_BY_NAME = {"Laplace_Eval": Laplace, "Laplace": Laplace,
            "Modified_Helmholtz_Eval": ModifiedHelmholtz, "ModifiedHelmholtz": ModifiedHelmholtz}
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
