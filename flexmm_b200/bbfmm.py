"""Black-box (Chebyshev) FMM: BB_FMM and BB_Helper (flexmm/flexmm2d/bbfmm.py).

A box's expansions are the p x p Chebyshev coefficients of the field on the
box scaled to [-1, 1]^2.  The operators, formed here on the host in FP64 as
the reference forms them, are:

* the Chebyshev nodes of the first kind (numpy's ``chebgauss``, reversed) on
  a p x p tensor grid and VI, the inverse of their 2-D Chebyshev Vandermonde
  matrix (bbfmm.py:133-143);
* M2MC = W2 . blockdiag(VI^T) with W2 the Vandermonde matrix of the four
  children's nodes in the parent's coordinates; L2LC = M2MC^T (bbfmm.py:145-161);
  level independent;
* per box width and offset, M2L = VI . K(nodes + offset w, nodes) . VI^T,
  compressed by the same SVD rule as the KIFMM operators (bbfmm.py:101-122,
  flexmm/flexmm2d/helpers.py:5-33).

The device runs S2M (Chebyshev moments), M2M, M2L, L2L (FP64 tensor-core
row GEMMs with fused gathers, ``csrc/rowgemm.cuh``), L2T (2-D Chebyshev
series) and P2P in FP64 (``csrc/bbfmm.cu``).
"""
import ctypes

import numpy as np

from . import _lib
from .helpers import SVD_TOL, offsets, width_key
from .kifmm import KI_FMM


def cheb_info(p):
    """Nodes, VI and M2MC of Chebyshev order p (BB_Helper.prepare, bbfmm.py:133-167)."""
    cheb = np.polynomial.chebyshev
    v = cheb.chebgauss(p)[0][::-1]
    nodex, nodey = np.meshgrid(v, v, indexing="ij")
    nodex, nodey = nodex.ravel(), nodey.ravel()
    V = cheb.chebvander2d(nodex, nodey, [p - 1, p - 1])
    VI = np.linalg.inv(V)
    sx, sy = nodex / 2, nodey / 2
    cx = np.concatenate([sx - 0.5, sx - 0.5, sx + 0.5, sx + 0.5])
    cy = np.concatenate([sy - 0.5, sy + 0.5, sy - 0.5, sy + 0.5])
    n = p * p
    W1 = np.zeros((4 * n, 4 * n))
    for i in range(4):
        W1[i * n:(i + 1) * n, i * n:(i + 1) * n] = VI.T
    W2 = cheb.chebvander2d(cx, cy, [p - 1, p - 1]).T
    M2MC = W2.dot(W1)
    return dict(nodex=nodex, nodey=nodey, VI=VI, M2MC=np.ascontiguousarray(M2MC))


class BBPrecomputation:
    """The 40 M2L operators of one width (BB_Precomputation, bbfmm.py:95-128)."""

    def __init__(self, width, p, kernel, info):
        self.width = width
        n = p * p
        VI = info["VI"]
        snx = info["nodex"] * 0.5 * width
        sny = info["nodey"] * 0.5 * width

        def form(sx, sy, tx, ty):  # out[j, i] = K(s_i, t_j)
            return np.ascontiguousarray(kernel.host(sx[None, :], sy[None, :], tx[:, None], ty[:, None]),
                                        dtype=np.float64)

        self.m2l_rank = np.zeros(len(offsets()), dtype=np.int32)
        self.m2l_a, self.m2l_b = [], []
        for o, (ox, oy) in enumerate(offsets()):
            m = VI.dot(form(snx + ox * width, sny + oy * width, snx, sny)).dot(VI.T)
            Um, Sm, VHm = np.linalg.svd(m)
            cuts = np.flatnonzero(Sm > SVD_TOL)
            if cuts.size == 0:
                self.m2l_a.append(None)
                self.m2l_b.append(None)
                continue
            r = int(cuts[-1]) + 1
            if 2 * r < n:
                self.m2l_rank[o] = r
                self.m2l_a.append(np.ascontiguousarray(Um[:, :r]))
                self.m2l_b.append(np.ascontiguousarray(VHm[:r] * Sm[:r, None]))
            else:
                self.m2l_rank[o] = -1
                self.m2l_a.append(np.ascontiguousarray(m))
                self.m2l_b.append(None)

    def upload(self, ops_handle):
        dp = ctypes.POINTER(ctypes.c_double)

        def ptr(a):
            return a.ctypes.data_as(dp) if a is not None else ctypes.cast(None, dp)

        arr_a = (dp * len(self.m2l_a))(*[ptr(a) for a in self.m2l_a])
        arr_b = (dp * len(self.m2l_b))(*[ptr(b) for b in self.m2l_b])
        lv = _lib.BBLevelOps(width=self.width,
                             m2l_rank=self.m2l_rank.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                             m2l_a=arr_a, m2l_b=arr_b)
        lid = ctypes.c_int(-1)
        _lib.call("fmm_bb_ops_add", ops_handle, ctypes.byref(lv), ctypes.byref(lid))
        return lid.value


class _BBOpsSet:
    def __init__(self, kernel, p, m2mc):
        h = ctypes.c_void_p()
        params = (ctypes.c_double * 4)(*kernel.params)
        _lib.call("fmm_bb_ops_create", kernel.kernel_id, params, p,
                  m2mc.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), ctypes.byref(h))
        self.handle = h

    def __del__(self):
        try:
            if self.handle is not None and _lib._LIB is not None:
                _lib._LIB.fmm_ops_destroy(self.handle)
        except Exception:
            pass
        self.handle = None


class BB_Helper:
    """Operator cache for one (kernel, p) (BB_Helper, bbfmm.py:130-210)."""

    def __init__(self, helper=None):
        self.kernel = None
        self.nequiv = None
        self.p = None
        self.info = None
        self.precomputations = {}
        self._level_ids = {}
        self._ops = None
        if helper is not None:
            self.__dict__ = helper.__dict__

    def attach(self, kernel, nequiv):
        p = int(round(np.sqrt(nequiv)))
        if self.kernel is None:
            self.kernel, self.nequiv, self.p = kernel, nequiv, p
            self.info = cheb_info(p)
        elif self.kernel.key != kernel.key or self.nequiv != nequiv:
            raise ValueError(f"helper holds operators for {self.kernel} with p={self.p}; "
                             f"got {kernel} with p={p}")

    def ops_set(self):
        if self._ops is None:
            self._ops = _BBOpsSet(self.kernel, self.p, self.info["M2MC"])
        return self._ops

    def collect_widths(self):
        return np.array(list(self.precomputations), dtype=float)

    def get_bbox(self, px, py, bbox):
        """Square bbox, snapped to a cached width (flexmm/flexmm2d/helpers.py:52-72)."""
        if bbox is None:
            bbox = [float(np.min(px)), float(np.max(px)), float(np.min(py)), float(np.max(py))]
        widths = self.collect_widths()
        if len(widths) > 0:
            small = np.min(widths)
            bw = max(bbox[1] - bbox[0], bbox[3] - bbox[2])
            width = 2 ** np.ceil(np.log2(bw / small)) * small
        else:
            width = max(bbox[1] - bbox[0], bbox[3] - bbox[2])
        cx = (bbox[1] + bbox[0]) / 2
        cy = (bbox[3] + bbox[2]) / 2
        return [float(cx - width / 2), float(cx + width / 2), float(cy - width / 2), float(cy + width / 2)]

    def level_id(self, width):
        key = width_key(width)
        if key not in self.precomputations:
            self.precomputations[key] = BBPrecomputation(width, self.p, self.kernel, self.info)
        if key not in self._level_ids:
            self._level_ids[key] = self.precomputations[key].upload(self.ops_set().handle)
        return self._level_ids[key]

    def get_precomputation(self, width):
        return self.precomputations[width_key(width)]


_DEFAULT_BB_HELPERS = {}


def default_bb_helper(kernel, nequiv):
    key = (kernel.key, nequiv)
    if key not in _DEFAULT_BB_HELPERS:
        _DEFAULT_BB_HELPERS[key] = BB_Helper()
    return _DEFAULT_BB_HELPERS[key]


class BB_FMM(KI_FMM):
    """Black-box FMM (BB_FMM, flexmm/flexmm2d/bbfmm.py:212-231): Chebyshev order p,
    p^2 coefficients per box, FP64.  Evaluation as KI_FMM's (source_evaluation,
    target_evaluation; potentials)."""

    _helper_cls = BB_Helper
    _max_nequiv = _lib.BB_MAX_P ** 2

    @staticmethod
    def _default_helper(kernel, nequiv):
        return default_bb_helper(kernel, nequiv)

    def __init__(self, x, y, kernel_eval, Ncutoff=50, p=8, dtype=float, bbox=None, helper=None,
                 verbose=False, **kernel_params):
        if not 2 <= p <= _lib.BB_MAX_P:
            raise ValueError(f"p must be in [2, {_lib.BB_MAX_P}]")
        self.p = int(p)
        super().__init__(x, y, kernel_eval, Ncutoff, self.p ** 2, dtype=dtype, bbox=bbox,
                         helper=helper, verbose=verbose, precision="fp64", **kernel_params)
