"""Stokes FMM (flexmm/kifmm2d/vector/stokes_fmm.py:550-858).

A kernel-independent FMM for the 2-D Stokeslet: forces (taux, tauy) at the
sources, velocity (u, v) and pressure p at the targets.  A box carries
2 Nequiv equivalent forces on a circle plus one extra unknown of the
pressure-corrected forms (2 Nequiv + 1 values); the operators, formed here on
the host in FP64 as the reference forms them (Stokes_Kernel_Form,
Corrected_Stokes_Kernel_Form, Precomputation, stokes_fmm.py:472-591), are
uploaded once per box width, and the passes run on the GPU
(``csrc/stokes.cu``).

Differences from the reference, both result-preserving:

* ``bbox=None`` without precomputations, where the reference's Tree fails,
  takes the square around the points (the scalar FMMs' rule);
* the operators per width are cached in ``precomputations`` (pass the dict
  of a previous FMM to reuse them, as the reference's ``precomputations=``).
"""
import ctypes
import hashlib
import os

import numpy as np

from . import _lib
from .helpers import offsets, width_key
from .kifmm import _as_kind, _device_f64, _stream, _torch

SVD_TOL = 1e-15   # SVD_Solver, stokes_fmm.py:541
M2L_TOL = 1e-14   # M2L_Evaluator cut-off, stokes_fmm.py:586


def circles(width, theta):
    """Small and large circles of a box (get_level_information, stokes_fmm.py:17-27)."""
    dd = 0.1
    r1 = 0.5 * width * (np.sqrt(2) + dd)
    r2 = 0.5 * width * (4 - np.sqrt(2) - 2 * dd)
    return r1 * np.cos(theta), r1 * np.sin(theta), r2 * np.cos(theta), r2 * np.sin(theta)


def stokes_form(sx, sy, tx, ty, corrected=False):
    """Forces at s -> (u, v at t; p at the mean of t) (Stokes_Kernel_Form /
    Corrected_Stokes_Kernel_Form, stokes_fmm.py:472-539)."""
    ns, nt = sx.size, tx.size
    fscale = 0.25 / np.pi
    pscale = 2 * fscale
    G = np.zeros((2 * nt + 1, 2 * ns + (1 if corrected else 0)))
    dx = tx[:, None] - sx[None, :]
    dy = ty[:, None] - sy[None, :]
    id2 = 1.0 / (dx * dx + dy * dy)
    logid = 0.5 * np.log(id2)
    G[:nt, :ns] = fscale * (logid + dx * dx * id2)
    G[nt:2 * nt, :ns] = fscale * dx * dy * id2
    G[:nt, ns:2 * ns] = fscale * dx * dy * id2
    G[nt:2 * nt, ns:2 * ns] = fscale * (logid + dy * dy * id2)
    px = np.mean(tx) - sx
    py = np.mean(ty) - sy
    pid2 = 1.0 / (px * px + py * py)
    prow = pscale * np.concatenate([px * pid2, py * pid2])
    if corrected:
        G[-1, :-1] = prow
        G[:-1, -1] = prow
    else:
        G[-1, :] = prow
    return G


class _SVD:
    """U, 1/S (0 below tol), VH of an SVD solve (SVD_Solver, stokes_fmm.py:540-549)."""

    def __init__(self, A, tol=SVD_TOL):
        self.U, S, self.VH = np.linalg.svd(A)
        with np.errstate(divide="ignore"):
            self.SI = np.where(S < tol, 0.0, 1.0 / S)


class StokesPrecomputation:
    """Operators of one box width (Precomputation, stokes_fmm.py:550-591)."""

    def __init__(self, width, nequiv):
        self.width = width
        self.Nequiv = nequiv
        theta = np.linspace(0, 2 * np.pi, nequiv, endpoint=False)
        sx, sy, lx, ly = circles(width, theta)
        self.small_x, self.small_y = sx, sy
        self.large_x, self.large_y = np.ascontiguousarray(lx), np.ascontiguousarray(ly)
        self.e2c = _SVD(stokes_form(sx, sy, lx, ly, corrected=True))
        self.c2e = _SVD(stokes_form(lx, ly, sx, sy, corrected=True))
        ssx, ssy, _, _ = circles(0.5 * width, theta)
        q = 0.25 * width
        shifts = [(-q, -q), (-q, q), (q, -q), (q, q)]
        self.m2mc = np.ascontiguousarray(np.column_stack(
            [stokes_form(ssx + a, ssy + b, lx, ly) for a, b in shifts]))
        self.l2lc = np.ascontiguousarray(np.vstack(
            [stokes_form(lx, ly, ssx + a, ssy + b) for a, b in shifts]))
        n1 = 2 * nequiv + 1
        self.m2l_rank = np.zeros(len(offsets()), dtype=np.int32)
        self.m2l_a, self.m2l_b = [], []
        for ox, oy in offsets():
            m = stokes_form(sx + ox * width, sy + oy * width, sx, sy)
            U, S, VH = np.linalg.svd(m)
            cuts = np.flatnonzero(S > M2L_TOL)
            if cuts.size == 0:
                self.m2l_a.append(None)
                self.m2l_b.append(None)
                continue
            r = int(cuts[-1]) + 1
            if r < n1:   # M2L_Evaluator: factors when the cut-off is below the row count
                self.m2l_rank[len(self.m2l_a)] = r
                self.m2l_a.append(np.ascontiguousarray(U[:, :r]))
                self.m2l_b.append(np.ascontiguousarray(VH[:r] * S[:r, None]))
            else:
                self.m2l_rank[len(self.m2l_a)] = -1
                self.m2l_a.append(np.ascontiguousarray(m))
                self.m2l_b.append(None)

    def upload(self, ops_handle):
        dp = ctypes.POINTER(ctypes.c_double)

        def ptr(a):
            return np.ascontiguousarray(a).ctypes.data_as(dp) if a is not None else ctypes.cast(None, dp)

        keep = [np.ascontiguousarray(a) for a in (self.e2c.U, self.e2c.SI, self.e2c.VH,
                                                 self.c2e.U, self.c2e.SI, self.c2e.VH)]
        arr_a = (dp * len(self.m2l_a))(*[ptr(a) for a in self.m2l_a])
        arr_b = (dp * len(self.m2l_b))(*[ptr(b) for b in self.m2l_b])
        lv = _lib.StokesLevelOps(
            width=self.width, large_x=ptr(self.large_x), large_y=ptr(self.large_y),
            e2c_u=ptr(keep[0]), e2c_sinv=ptr(keep[1]), e2c_vh=ptr(keep[2]),
            c2e_u=ptr(keep[3]), c2e_sinv=ptr(keep[4]), c2e_vh=ptr(keep[5]),
            m2mc=ptr(self.m2mc), l2lc=ptr(self.l2lc),
            m2l_rank=self.m2l_rank.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
            m2l_a=arr_a, m2l_b=arr_b)
        lid = ctypes.c_int(-1)
        _lib.call("fmm_stokes_ops_add", ops_handle, ctypes.byref(lv), ctypes.byref(lid))
        return lid.value


    def to_arrays(self):
        """The operators as named arrays (one .npz file of the on-disk cache)."""
        d = dict(width=np.float64(self.width), nequiv=np.int64(self.Nequiv),
                 small_x=self.small_x, small_y=self.small_y, large_x=self.large_x,
                 large_y=self.large_y, m2mc=self.m2mc, l2lc=self.l2lc, m2l_rank=self.m2l_rank)
        for name in ("e2c", "c2e"):
            svd = getattr(self, name)
            d[f"{name}_U"], d[f"{name}_SI"], d[f"{name}_VH"] = svd.U, svd.SI, svd.VH
        for o, (a, b) in enumerate(zip(self.m2l_a, self.m2l_b)):
            if a is not None:
                d[f"m2l_a_{o}"] = a
            if b is not None:
                d[f"m2l_b_{o}"] = b
        return d

    @classmethod
    def from_arrays(cls, d):
        """Inverse of to_arrays (no operator is recomputed)."""
        pre = cls.__new__(cls)
        pre.width = float(d["width"])
        pre.Nequiv = int(d["nequiv"])
        for name in ("small_x", "small_y", "large_x", "large_y", "m2mc", "l2lc"):
            setattr(pre, name, np.ascontiguousarray(d[name], dtype=np.float64))
        for name in ("e2c", "c2e"):
            svd = _SVD.__new__(_SVD)
            svd.U, svd.SI, svd.VH = (np.asarray(d[f"{name}_{k}"], dtype=np.float64)
                                     for k in ("U", "SI", "VH"))
            setattr(pre, name, svd)
        pre.m2l_rank = np.ascontiguousarray(d["m2l_rank"], dtype=np.int32)
        pre.m2l_a, pre.m2l_b = [], []
        for o in range(len(pre.m2l_rank)):
            a, b = d.get(f"m2l_a_{o}"), d.get(f"m2l_b_{o}")
            pre.m2l_a.append(None if a is None else np.ascontiguousarray(a, dtype=np.float64))
            pre.m2l_b.append(None if b is None else np.ascontiguousarray(b, dtype=np.float64))
        return pre


def stokes_precomputation(width, nequiv, cache_dir=None):
    """Operators of one width: from the on-disk cache (``cache_dir`` or the
    environment variable FLEXMM_B200_CACHE) when it holds them, else formed
    and then written there (one .npz per width under a directory named by
    Nequiv and the file format's version)."""
    from .helpers import CACHE_VERSION
    cache_dir = cache_dir if cache_dir is not None else os.environ.get("FLEXMM_B200_CACHE")
    path = None
    if cache_dir:
        tag = hashlib.sha1(repr(("stokes", int(nequiv), CACHE_VERSION)).encode()).hexdigest()[:20]
        d = os.path.join(cache_dir, "stokes_" + tag)
        path = os.path.join(d, f"w_{width_key(width)!r}.npz")
        try:
            with np.load(path) as z:
                pre = StokesPrecomputation.from_arrays({k: z[k] for k in z.files})
            if pre.Nequiv == nequiv and width_key(pre.width) == width_key(width):
                return pre
        except Exception:
            pass  # absent, damaged or half-written: formed again below
    pre = StokesPrecomputation(width, nequiv)
    if path:
        from .helpers import save_npz_atomic
        save_npz_atomic(path, pre.to_arrays())
    return pre


class _StokesOps:
    def __init__(self, nequiv):
        h = ctypes.c_void_p()
        _lib.call("fmm_stokes_ops_create", nequiv, ctypes.byref(h))
        self.handle = h
        self.level_ids = {}

    def __del__(self):
        try:
            if self.handle is not None and _lib._LIB is not None:
                _lib._LIB.fmm_ops_destroy(self.handle)
        except Exception:
            pass
        self.handle = None


class FMM:
    """Stokes FMM (FMM, stokes_fmm.py:592-858): ``FMM(x, y, Nequiv, Ncutoff, bbox)``,
    ``precompute()``, ``build_expansions(taux, tauy)``,
    ``evaluate_to_points(x, y, check_self) -> (u, v, p)``."""

    def __init__(self, x, y, Nequiv=48, Ncutoff=50, bbox=None, precomputations=None, verbose=False):
        if Nequiv > _lib.MAX_NEQUIV:
            raise ValueError(f"Nequiv must be <= {_lib.MAX_NEQUIV}")
        _lib.load()
        from .kernels import Stokes
        self.kernel = Stokes()   # the registered "Stokes" kernel
        self.Nequiv = int(Nequiv)
        self.Ncutoff = int(Ncutoff)
        self.verbose = verbose
        self.input_precomputations = precomputations
        xd, _ = _device_f64(x)
        yd, _ = _device_f64(y)
        if xd.numel() != yd.numel():
            raise ValueError("x and y differ in length")
        self.N = int(xd.numel())
        self._x, self._y = xd, yd
        self.bbox = self._adjust_bbox(xd, yd, bbox, precomputations)
        plan = ctypes.c_void_p()
        ops = (precomputations or {}).get("__ops__") if isinstance(precomputations, dict) else None
        self._ops = ops if ops is not None else _StokesOps(self.Nequiv)
        bb = (ctypes.c_double * 4)(*self.bbox)
        _lib.call("fmm_plan_create", self._ops.handle, ctypes.c_void_p(xd.data_ptr()),
                  ctypes.c_void_p(yd.data_ptr()), self.N, self.Ncutoff, bb, _stream(),
                  ctypes.byref(plan))
        self._plan = plan
        nl = ctypes.c_int()
        widths = (ctypes.c_double * _lib.MAX_LEVELS)()
        _lib.call("fmm_plan_info", plan, ctypes.byref(nl), widths, None)
        self._widths = [widths[i] for i in range(nl.value)]
        self.precomputations = None

    @staticmethod
    def _adjust_bbox(xd, yd, bbox, precomputations):
        """Square bbox snapped to known widths (adjust_bbox, stokes_fmm.py:608-637)."""
        if bbox is None:
            bbox = [xd.min().item(), xd.max().item(), yd.min().item(), yd.max().item()]
            square = True
        else:
            bbox = [float(v) for v in bbox]
            square = precomputations is not None
        if not square:
            return bbox
        widths = [w for w in (precomputations or {}) if w != "__ops__"]
        bw = max(bbox[1] - bbox[0], bbox[3] - bbox[2])
        if widths:
            small = min(widths)
            width = 2 ** np.ceil(np.log2(bw / small)) * small
        else:
            width = bw
        cx, cy = (bbox[1] + bbox[0]) / 2, (bbox[3] + bbox[2]) / 2
        return [cx - width / 2, cx + width / 2, cy - width / 2, cy + width / 2]

    def precompute(self):
        """Operators for every level width (precompute, stokes_fmm.py:644-657)."""
        pre = dict(self.input_precomputations or {})
        pre["__ops__"] = self._ops
        for m, w in enumerate(self._widths):
            key = width_key(w)
            if key not in pre:
                pre[key] = stokes_precomputation(w, self.Nequiv)
            if key not in self._ops.level_ids:
                self._ops.level_ids[key] = pre[key].upload(self._ops.handle)
            _lib.call("fmm_plan_bind", self._plan, m, self._ops.level_ids[key])
        self.precomputations = pre

    def build_expansions(self, taux, tauy):
        if self.precomputations is None:
            self.precompute()
        fx, _ = _device_f64(taux)
        fy, _ = _device_f64(tauy)
        if fx.numel() != self.N or fy.numel() != self.N:
            raise ValueError(f"forces must have {self.N} entries")
        _lib.call("fmm_build_expansions2", self._plan, ctypes.c_void_p(fx.data_ptr()),
                  ctypes.c_void_p(fy.data_ptr()), _stream())
        self._tau = (fx, fy)

    def build_expansions_dipole(self, taux, tauy, sigmax, sigmay, dipx, dipy):
        """Forces plus stresslets (double layer of strength (sigmax, sigmay)
        along the normals (dipx, dipy)): build_expansions_dipole,
        stokes_fmm.py:738-826.  Later evaluations include the stresslets."""
        if self.precomputations is None:
            self.precompute()
        arrs = [_device_f64(a)[0] for a in (taux, tauy, sigmax, sigmay, dipx, dipy)]
        if any(a.numel() != self.N for a in arrs):
            raise ValueError(f"every array must have {self.N} entries")
        _lib.call("fmm_build_expansions2_dipole", self._plan,
                  *[ctypes.c_void_p(a.data_ptr()) for a in arrs], _stream())
        self._tau = tuple(arrs)

    def evaluate_to_points_dipole(self, x, y, check_self=False):
        """(u, v, p) at (x, y) after build_expansions_dipole
        (evaluate_to_points_dipole, stokes_fmm.py:844-858)."""
        return self.evaluate_to_points(x, y, check_self)

    def evaluate_to_points(self, x, y, check_self=False):
        """(u, v, p) at (x, y); ``check_self`` skips coincident sources."""
        torch = _torch()
        xd, kind = _device_f64(x)
        yd, _ = _device_f64(y)
        m = xd.numel()
        out = torch.empty((3, m), dtype=torch.float64, device="cuda")
        _lib.call("fmm_evaluate_outputs", self._plan, _lib.EVALUATORS["stokes"][0],
                  ctypes.c_void_p(xd.data_ptr()), ctypes.c_void_p(yd.data_ptr()), m,
                  1 if check_self else 0, ctypes.c_void_p(out.data_ptr()), m, _stream())
        res = _as_kind(out, kind, (3, m))
        return res[0], res[1], res[2]

    def status(self):
        _lib.call("fmm_plan_status", self._plan)

    def __del__(self):
        try:
            if getattr(self, "_plan", None) is not None and _lib._LIB is not None:
                _lib._LIB.fmm_plan_destroy(self._plan)
        except Exception:
            pass
        self._plan = None
