"""Near-field-only evaluation: the LocalEvaluator family.

The reference's LocalEvaluator (flexmm/flexmm2d/local_evaluator.py) sums a
kernel over the sources of a target leaf's colleagues only -- no expansions,
no far field -- on a LocalTree (flexmm/local_tree.py): the FMM's quadtree
except that a box splits only while it holds more than ``ncutoff`` points
AND is wider than twice ``min_distance``, so every source within
``min_distance`` of a target sits in a colleague of the target's leaf.  It
is meant for kernels that vanish (or are dropped) beyond ``min_distance``.

Here the tree and the colleague sum run on the GPU
(fmm_plan_create_local / fmm_local_evaluate): the FMM's tree build with
the width floor, and the P2P kernel of the evaluation with the far field
off.  The kernel is a registered device kernel (a name such as
'Laplace_Eval', or a ``Kernel``, e.g. a compactly supported radial one from
``flexmm_b200.kernels.radial``); the reference takes a numba
``Kernel_Add(sx, sy, tx, ty, tau, out)`` that adds K(s, t) tau to out[0].

Category and periodic variants: ``flexmm_b200.local_evaluator_category``,
``flexmm_b200.periodic_local_evaluator_category``.
"""
import ctypes

import numpy as np

from . import _lib
from .kernels import resolve
from .kifmm import _as_kind, _device_f64, _stream, _torch

_OPS = {}   # kernel key -> operator set (kernel identity and parameters only)


def _ops_for(kernel):
    if kernel.key not in _OPS:
        h = ctypes.c_void_p()
        params = (ctypes.c_double * 4)(*kernel.params)
        _lib.call("fmm_ops_create", kernel.kernel_id, params, 1, ctypes.byref(h))
        _OPS[kernel.key] = h
    return _OPS[kernel.key]


class LocalHelper:
    """The reference's LocalHelper (local_evaluator.py:17-30): the bbox of the
    points when none is given (not squared: the tree's root box takes the x
    extent as its width, as LocalTree does)."""

    functions = {}

    def __init__(self, helper=None):
        pass

    def get_bbox(self, px, py, bbox):
        if bbox is None:
            px = np.asarray(px)
            py = np.asarray(py)
            bbox = [float(np.min(px)), float(np.max(px)), float(np.min(py)), float(np.max(py))]
        return [float(v) for v in bbox]


def _host(a):
    torch = _torch()
    if isinstance(a, torch.Tensor):
        return a.detach().cpu().numpy()
    return np.asarray(a)


class _LocalCore:
    """Tree + near-field sums; shared by the three evaluator classes."""

    def _setup(self, x, y, kernel_eval, min_distance, ncutoff, bbox, helper, kernel_params):
        _lib.load()
        self.kernel = resolve(kernel_eval, **kernel_params)
        if self.kernel.vector:
            raise ValueError("local evaluators take scalar kernels")
        self.min_distance = float(min_distance)
        self.ncutoff = int(ncutoff)
        self.helper = LocalHelper() if helper is None else helper
        self.bbox = self.helper.get_bbox(_host(x), _host(y), bbox)
        xd, _ = _device_f64(x)
        yd, _ = _device_f64(y)
        if xd.numel() != yd.numel():
            raise ValueError("x and y differ in length")
        self.N = int(xd.numel())
        self._x, self._y = xd, yd
        self._ops = _ops_for(self.kernel)
        plan = ctypes.c_void_p()
        bb = (ctypes.c_double * 4)(*self.bbox)
        _lib.call("fmm_plan_create_local", self._ops, ctypes.c_void_p(xd.data_ptr()),
                  ctypes.c_void_p(yd.data_ptr()), self.N, self.ncutoff, self.min_distance, bb,
                  _stream(), ctypes.byref(plan))
        self._plan = plan
        self._tau = None
        self._scat = None

    def load_tau(self, tau):
        td, _ = _device_f64(tau)
        if td.numel() != self.N:
            raise ValueError(f"tau has {td.numel()} entries, expected {self.N}")
        self._tau = td

    def _near(self, x, y, check, tcat=None):
        if self._tau is None:
            raise RuntimeError("load_tau has not run")
        torch = _torch()
        xd, kind = _device_f64(x)
        yd, _ = _device_f64(y)
        m = xd.numel()
        res = torch.empty(m, dtype=torch.float64, device="cuda")
        sc = tc = None
        if tcat is not None:
            sc = self._scat
            tc = torch.as_tensor(_host(tcat), dtype=torch.int64).reshape(-1).cuda()
            if tc.numel() != m:
                raise ValueError("one category per target")
        _lib.call("fmm_local_evaluate", self._plan, ctypes.c_void_p(self._tau.data_ptr()),
                  ctypes.c_void_p(xd.data_ptr()), ctypes.c_void_p(yd.data_ptr()), m,
                  1 if check else 0, ctypes.c_void_p(sc.data_ptr()) if sc is not None else None,
                  ctypes.c_void_p(tc.data_ptr()) if tc is not None else None,
                  ctypes.c_void_p(res.data_ptr()), _stream())
        self._keep = (tc,)   # alive until the stream has read them
        return res, kind

    @staticmethod
    def _into(out, res, kind):
        """Write the sums into the caller's ``out`` (shape [m] or [m, 1]), as
        the reference's evaluate_to_points fills its out array in place."""
        torch = _torch()
        if out is None:
            return _as_kind(res, kind, (res.numel(),))
        if isinstance(out, torch.Tensor):
            out.copy_(res.reshape(out.shape).to(out.device, out.dtype))
        else:
            out[...] = res.cpu().numpy().reshape(out.shape)
        return out

    def __del__(self):
        try:
            if getattr(self, "_plan", None) is not None and _lib._LIB is not None:
                _lib._LIB.fmm_plan_destroy(self._plan)
        except Exception:
            pass
        self._plan = None


class LocalEvaluator(_LocalCore):
    """``LocalEvaluator(x, y, kernel_eval, min_distance, ncutoff=20,
    dtype=float, bbox=None, helper=None, verbose=False)``, then
    ``load_tau(tau)`` and ``source_evaluation(x, y, out)`` (coincident
    sources skipped) / ``target_evaluation(x, y, out)``
    (flexmm/flexmm2d/local_evaluator.py:93-140)."""

    def __init__(self, x, y, kernel_eval, min_distance, ncutoff=20, dtype=float, bbox=None,
                 helper=None, verbose=False, **kernel_params):
        if dtype not in (float, np.float64):
            raise NotImplementedError("only real float64 densities are supported")
        self.verbose = verbose
        self._setup(x, y, kernel_eval, min_distance, ncutoff, bbox, helper, kernel_params)

    def source_evaluation(self, x, y, out=None):
        return self.evaluate_to_points(x, y, "neighbor_potential_source_evaluation", out)

    def target_evaluation(self, x, y, out=None):
        return self.evaluate_to_points(x, y, "neighbor_potential_target_evaluation", out)

    def evaluate_to_points(self, x, y, name, out=None):
        if name not in ("neighbor_potential_source_evaluation", "neighbor_potential_target_evaluation"):
            raise KeyError(f"evaluator {name!r} is not registered")
        res, kind = self._near(x, y, name == "neighbor_potential_source_evaluation")
        return self._into(out, res, kind)
