"""Vectorised numpy twins of the reference's example kernels (oracle only).

Laplace_Eval follows examples/kifmm_laplace.py:24-29.
"""
import numpy as np


def laplace(sx, sy, tx, ty):
    dx = tx - sx
    dy = ty - sy
    d2 = dx * dx + dy * dy
    return -np.log(d2) / (4 * np.pi)


KERNELS = {"Laplace_Eval": laplace}
