"""Vectorised numpy twins of the reference's example kernels (oracle only).

Laplace_Eval follows examples/kifmm_laplace.py:24-29; Modified_Helmholtz_Eval
examples/kifmm_modified_helmholtz.py:33-39 with K0 from scipy.special (the
example tabulates the same function with function_generator).
"""
import numpy as np


def laplace(sx, sy, tx, ty):
    dx = tx - sx
    dy = ty - sy
    d2 = dx * dx + dy * dy
    return -np.log(d2) / (4 * np.pi)


def mod_helmholtz(k):
    from scipy.special import k0

    def kernel(sx, sy, tx, ty):
        dx = tx - sx
        dy = ty - sy
        return k0(k * np.sqrt(dx * dx + dy * dy)) / (2 * np.pi)
    return kernel


KERNELS = {"Laplace_Eval": laplace}
