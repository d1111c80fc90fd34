"""flexmm_b200: the 2D FMM evaluation path of dbstein/flexmm on NVIDIA B200.

Public surface (mirrors the reference's):

* ``KI_FMM``     kernel-independent FMM   (flexmm/flexmm2d/kifmm.py)
* ``KI_Helper``  per-width operator cache (flexmm/flexmm2d/helpers.py)
* ``BB_FMM``, ``BB_Helper``  black-box Chebyshev FMM (flexmm/flexmm2d/bbfmm.py)
* ``Laplace_Eval`` and the kernel registry (``flexmm_b200.kernels``)

The compute runs in ``flexmm_b200/_lib/libflexmm_b200.so`` (hand-written
sm_100a CUDA behind the C ABI in ``include/flexmm_b200.h``); build it with
``python -m flexmm_b200.build``.
"""
from .bbfmm import BB_FMM, BB_Helper
from .helpers import KI_Helper
from .kernels import Kernel, Laplace, resolve
from .kifmm import KI_FMM, direct_evaluation, enable_timing, read_timing, set_split_evaluation

Laplace_Eval = Laplace()

__all__ = ["KI_FMM", "KI_Helper", "BB_FMM", "BB_Helper", "Kernel", "Laplace", "Laplace_Eval", "resolve",
           "direct_evaluation", "enable_timing", "read_timing", "set_split_evaluation"]
