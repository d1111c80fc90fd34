"""Operator precomputation and caching (the reference's Helper / Precomputation).

Mirrors flexmm/flexmm2d/helpers.py:35-84 and flexmm/flexmm2d/kifmm.py:13-82:
per box width, the equivalent / check circles, the check-to-equivalent
solve, the M2M operator (whose transpose is L2L) and the 40 M2L operators,
SVD-compressed exactly as M2L_Evaluator does.  The operators are formed on
the host in FP64 with the kernel's numpy twin and uploaded once into a
device operator set (``fmm_ops``); plans bind their levels to entries.

Two deliberate differences from the reference:

* the check-to-equivalent solve is stored as the SVD factors
  (U, 1/S, VH) and applied on the GPU as two GEMMs and a scaling, as in
  flexmm/kifmm2d/scalar/helpers.py:240-248, instead of LU (the two agree to
  ~1e-15; an explicit inverse would not);
* a helper is bound to one (kernel, Nequiv): passing it to an FMM with a
  different kernel or Nequiv raises, instead of silently reusing the first
  kernel's operators (the shared default ``helper=KI_Helper()`` of
  flexmm/flexmm2d/kifmm.py:123).  With ``helper=None`` a process-wide helper
  per (kernel, params, Nequiv) is used, so operators stay warm across objects.
"""
import ctypes
import hashlib
import os

import numpy as np

from . import _lib

CACHE_VERSION = 1      # on-disk operator files: bump when their content changes

SVD_TOL = 1e-14        # M2L compression, flexmm/flexmm2d/helpers.py:197
C2E_TOL = 1e-15        # SVD_Solver, flexmm/kifmm2d/scalar/helpers.py:241


def width_key(width):
    """Cache key of a box width (FloatDict, flexmm/flexmm2d/float_dict.py:23-24)."""
    return round(width, 12)


def surfaces(width, theta):
    """Small (equivalent) and large (check) circles (flexmm/flexmm2d/kifmm.py:158-168)."""
    dd = 0.0
    r1 = 0.5 * width * (np.sqrt(2) + dd)
    r2 = 0.5 * width * (4 - np.sqrt(2) - 2 * dd)
    return r1 * np.cos(theta), r1 * np.sin(theta), r2 * np.cos(theta), r2 * np.sin(theta)


def offsets():
    """The 40 far-field offsets in device order (ox outer, oy inner)."""
    return [(a, b) for a in range(-3, 4) for b in range(-3, 4) if not (abs(a) <= 1 and abs(b) <= 1)]


class KIPrecomputation:
    """Operators of one width (KI_Precomputation, flexmm/flexmm2d/kifmm.py:13-62)."""

    def __init__(self, width, nequiv, kernel):
        self.width = width
        n = nequiv
        theta = np.linspace(0, 2 * np.pi, n, endpoint=False)

        def form(sx, sy, tx, ty):  # out[j, i] = K(s_i, t_j)
            return np.ascontiguousarray(kernel.host(sx[None, :], sy[None, :], tx[:, None], ty[:, None]),
                                        dtype=np.float64)

        sx, sy, lx, ly = surfaces(width, theta)
        s2l = form(sx, sy, lx, ly)
        U, S, VH = np.linalg.svd(s2l)
        with np.errstate(divide="ignore"):
            self.c2e_sinv = np.where(S < C2E_TOL, 0.0, 1.0 / S)
        self.c2e_u = np.ascontiguousarray(U)
        self.c2e_vh = np.ascontiguousarray(VH)
        ssx, ssy, _, _ = surfaces(0.5 * width, theta)
        q = 0.25 * width
        cex = np.concatenate([ssx - q, ssx - q, ssx + q, ssx + q])
        cey = np.concatenate([ssy - q, ssy + q, ssy - q, ssy + q])
        self.m2mc = form(cex, cey, lx, ly)
        self.small_x, self.small_y = sx, sy
        self.large_x, self.large_y = np.ascontiguousarray(lx), np.ascontiguousarray(ly)
        # M2L_Evaluator semantics (flexmm/flexmm2d/helpers.py:5-33)
        self.m2l_rank = np.zeros(len(offsets()), dtype=np.int32)
        self.m2l_a = []
        self.m2l_b = []
        for o, (ox, oy) in enumerate(offsets()):
            m = form(sx + ox * width, sy + oy * width, sx, sy)
            Um, Sm, VHm = np.linalg.svd(m)
            cuts = np.flatnonzero(Sm > SVD_TOL)
            if cuts.size == 0:
                self.m2l_rank[o] = 0
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
                self.m2l_a.append(m)
                self.m2l_b.append(None)

    def to_arrays(self):
        """The operators as named arrays (one .npz file of the on-disk cache)."""
        d = dict(width=np.float64(self.width), c2e_sinv=self.c2e_sinv, c2e_u=self.c2e_u,
                 c2e_vh=self.c2e_vh, m2mc=self.m2mc, small_x=self.small_x, small_y=self.small_y,
                 large_x=self.large_x, large_y=self.large_y, m2l_rank=self.m2l_rank)
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
        for name in ("c2e_sinv", "c2e_u", "c2e_vh", "m2mc", "small_x", "small_y", "large_x",
                     "large_y"):
            setattr(pre, name, np.ascontiguousarray(d[name], dtype=np.float64))
        pre.m2l_rank = np.ascontiguousarray(d["m2l_rank"], dtype=np.int32)
        pre.m2l_a, pre.m2l_b = [], []
        for o in range(len(pre.m2l_rank)):
            a, b = d.get(f"m2l_a_{o}"), d.get(f"m2l_b_{o}")
            pre.m2l_a.append(None if a is None else np.ascontiguousarray(a, dtype=np.float64))
            pre.m2l_b.append(None if b is None else np.ascontiguousarray(b, dtype=np.float64))
        return pre

    def upload(self, ops_handle):
        dp = ctypes.POINTER(ctypes.c_double)

        def ptr(a):
            return a.ctypes.data_as(dp) if a is not None else ctypes.cast(None, dp)

        arr_a = (dp * len(self.m2l_a))(*[ptr(a) for a in self.m2l_a])
        arr_b = (dp * len(self.m2l_b))(*[ptr(b) for b in self.m2l_b])
        lv = _lib.LevelOps(
            width=self.width, large_x=ptr(self.large_x), large_y=ptr(self.large_y),
            c2e_u=ptr(self.c2e_u), c2e_sinv=ptr(self.c2e_sinv), c2e_vh=ptr(self.c2e_vh),
            m2mc=ptr(self.m2mc),
            m2l_rank=self.m2l_rank.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
            m2l_a=arr_a, m2l_b=arr_b)
        lid = ctypes.c_int(-1)
        _lib.call("fmm_ops_add", ops_handle, ctypes.byref(lv), ctypes.byref(lid))
        return lid.value


class OpsSet:
    """Owner of one device operator set (``fmm_ops``); destroyed with its last reference."""

    def __init__(self, kernel, nequiv):
        h = ctypes.c_void_p()
        params = (ctypes.c_double * 4)(*kernel.params)
        _lib.call("fmm_ops_create", kernel.kernel_id, params, nequiv, ctypes.byref(h))
        self.handle = h

    def __del__(self):
        try:
            if self.handle is not None and _lib._LIB is not None:
                _lib._LIB.fmm_ops_destroy(self.handle)
        except Exception:
            pass
        self.handle = None


class _NamedForm:
    """A placeholder for one of the reference helper's compiled functions
    (helper.functions[...]): only its name matters here, the device forms are
    built in (register_evaluator / register_upwardor match it by name)."""

    def __init__(self, name):
        self.__name__ = name

    def __repr__(self):
        return f"<built-in {self.__name__}>"


class KI_Helper:

    """Operator cache for one (kernel, Nequiv) (Helper, flexmm/flexmm2d/helpers.py:35-84).

    ``cache_dir`` (or the environment variable FLEXMM_B200_CACHE) keeps the
    host operators on disk across processes, one .npz file per width under a
    directory named by (kernel, parameters, Nequiv, format version): a width
    the helper needs is read from there instead of formed, and every width it
    forms is written there.  Files are read only when their width is asked
    for, so bbox snapping sees the widths met in this process alone, as in
    the reference (the tree, and so the results, never depend on what an
    earlier run left on disk).  Tabulated kernels (``radial``) are not cached
    on disk: their identity is not in their parameters."""

    # the names of the reference helper's base functions that scripts pass
    # back to register_evaluator / register_upwardor
    # (flexmm/kifmm2d/scalar/helpers.py:113-124)
    functions = {n: _NamedForm(n) for n in ("kernel_app", "extra_kernel_app")}

    def __init__(self, helper=None, cache_dir=None):
        self.kernel = None
        self.nequiv = None
        self.precomputations = {}   # width_key -> KIPrecomputation
        self._level_ids = {}        # width_key -> device operator entry
        self._ops = None
        self.cache_dir = cache_dir if cache_dir is not None else os.environ.get("FLEXMM_B200_CACHE")
        if helper is not None:      # share the other helper's cache, like the reference
            self.__dict__ = helper.__dict__

    def attach(self, kernel, nequiv):
        if self.kernel is None:
            self.kernel = kernel
            self.nequiv = nequiv
        elif self.kernel.key != kernel.key or self.nequiv != nequiv:
            raise ValueError(f"helper holds operators for {self.kernel} with Nequiv={self.nequiv}; "
                             f"got {kernel} with Nequiv={nequiv}")

    def _disk_dir(self):
        from .kernels import KERNEL_RADIAL_TABLE
        if not self.cache_dir or self.kernel is None or self.kernel.kernel_id == KERNEL_RADIAL_TABLE:
            return None
        tag = repr((self.kernel.key, int(self.nequiv), CACHE_VERSION)).encode()
        return os.path.join(self.cache_dir, "ki_" + hashlib.sha1(tag).hexdigest()[:20])

    def _disk_path(self, key):
        d = self._disk_dir()
        return None if d is None else os.path.join(d, f"w_{key!r}.npz")

    def _load_disk(self, key):
        """The operators of one width from the disk cache, or None (absent,
        damaged, half-written by a crashed writer, or for another Nequiv)."""
        path = self._disk_path(key)
        if path is None or not os.path.isfile(path):
            return None
        try:
            with np.load(path) as z:
                pre = KIPrecomputation.from_arrays({k: z[k] for k in z.files})
        except Exception:
            return None  # that width is formed again
        if pre.c2e_u.shape[0] != self.nequiv or width_key(pre.width) != key:
            return None
        return pre

    def _save_disk(self, key, pre):
        path = self._disk_path(key)
        if path is not None:
            save_npz_atomic(path, pre.to_arrays())

    def ops_set(self):
        if self._ops is None:
            self._ops = OpsSet(self.kernel, self.nequiv)
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

    def precomputation(self, width):
        """The host operators of a width: from memory, the disk cache, or formed
        (and then written to the disk cache)."""
        key = width_key(width)
        if key not in self.precomputations:
            pre = self._load_disk(key)
            if pre is None:
                pre = KIPrecomputation(width, self.nequiv, self.kernel)
                self._save_disk(key, pre)
            self.precomputations[key] = pre
        return self.precomputations[key]

    def level_id(self, width):
        key = width_key(width)
        pre = self.precomputation(width)
        if key not in self._level_ids:
            self._level_ids[key] = pre.upload(self.ops_set().handle)
        return self._level_ids[key]

    def get_precomputation(self, width):
        return self.precomputations[width_key(width)]


def save_npz_atomic(path, arrays):
    """Write ``arrays`` to ``path`` (.npz) so that readers see the whole file or
    none: the data goes to a uniquely named temporary file in the same
    directory (a name no reader takes for a cache file), then replaces the
    target in one rename."""
    import tempfile
    d = os.path.dirname(path)
    os.makedirs(d, exist_ok=True)
    fd, tmp = tempfile.mkstemp(dir=d, prefix=".w_", suffix=".tmp")
    try:
        with os.fdopen(fd, "wb") as f:
            np.savez(f, **arrays)
        os.replace(tmp, path)
    except BaseException:
        try:
            os.unlink(tmp)
        except OSError:
            pass
        raise


_DEFAULT_HELPERS = {}


def default_helper(kernel, nequiv):
    key = (kernel.key, nequiv)
    if key not in _DEFAULT_HELPERS:
        _DEFAULT_HELPERS[key] = KI_Helper()
    return _DEFAULT_HELPERS[key]
