"""KI_FMM: the reference's kernel-independent FMM object, on a B200.

Same constructor, methods and results as flexmm/flexmm2d/kifmm.py:122-144
(with FMM, flexmm/flexmm2d/fmm.py:32-176)::

    F = KI_FMM(x, y, Laplace_Eval, Ncutoff, Nequiv, bbox=bbox, helper=helper)
    F.build_expansions(tau)
    u_src = F.source_evaluation(x, y)       # skips coincident source/target pairs
    u_tgt = F.target_evaluation(tx, ty)

Inputs may be numpy arrays (results come back as numpy) or torch tensors
(results stay torch tensors on the GPU).  ``precision="mixed"`` selects the
split-precision form (FP32 kernel evaluations, 3xTF32 tensor-core far-field
GEMMs, FP64 check-to-equivalent; Laplace, and the modified Helmholtz
potential); the default ``"fp64"`` matches the reference to 1e-12.  All work runs on the current CUDA
device and torch's current stream, through ``libflexmm_b200.so``; there is
no CPU path.
"""
import ctypes
import time

import numpy as np

from . import _lib
from .helpers import KI_Helper, default_helper
from .kernels import resolve


def _torch():
    import torch
    return torch


def _device_f64(a):
    """(device float64 contiguous 1-D tensor, kind) with kind in
    {"numpy", "cpu", "cuda"}: results are returned in the same kind."""
    torch = _torch()
    if isinstance(a, torch.Tensor):
        kind = "cuda" if a.is_cuda else "cpu"
        t = a.reshape(-1)
        if t.dtype != torch.float64 or not t.is_cuda or not t.is_contiguous():
            t = t.to(device="cuda", dtype=torch.float64, non_blocking=t.is_pinned()).contiguous()
        return t, kind
    arr = np.ascontiguousarray(np.asarray(a, dtype=np.float64).ravel())
    return torch.from_numpy(arr).to("cuda", non_blocking=False), "numpy"


_COPY_STREAMS = {}


def _device_f64_early(a):
    """_device_f64, except that a pinned float64 host tensor is copied on a
    copy stream of its own: the copy overlaps the work already queued on the
    current stream (the tree's last kernels, when the charges arrive), and
    the current stream waits for it before anything that follows."""
    torch = _torch()
    if not (isinstance(a, torch.Tensor) and not a.is_cuda and a.is_pinned()
            and a.dtype == torch.float64 and a.is_contiguous()):
        return _device_f64(a)
    dev = torch.cuda.current_device()
    cs = _COPY_STREAMS.get(dev)
    if cs is None:
        cs = _COPY_STREAMS[dev] = torch.cuda.Stream(device=dev)
    cur = torch.cuda.current_stream()
    with torch.cuda.stream(cs):
        t = torch.empty(a.numel(), dtype=torch.float64, device="cuda")
        t.copy_(a.reshape(-1), non_blocking=True)
    cur.wait_stream(cs)
    t.record_stream(cur)  # its memory is reused only after the current stream is done with it
    return t, "cpu"


def _as_kind(out, kind, shape):
    if kind == "numpy":
        return out.cpu().numpy().reshape(shape)
    if kind == "cpu":
        host = _torch().empty(out.shape, dtype=out.dtype, pin_memory=True)
        host.copy_(out)
        return host
    return out


def _stream():
    return ctypes.c_void_p(_torch().cuda.current_stream().cuda_stream)


class TreeLevel:
    """One level of the GPU tree, with the reference's Level field names (flexmm/tree.py:275-360)."""


class TreeView:
    """Host copy of the GPU tree, shaped like the reference's Tree (flexmm/tree.py:447-589)."""

    def __init__(self, fmm):
        plan = fmm._plan
        L, widths, counts = fmm._levels, fmm._widths, fmm._counts
        T = int(sum(counts))
        xmin = np.empty(T)
        ymin = np.empty(T)
        bot = np.empty(T, np.int32)
        top = np.empty(T, np.int32)
        parent = np.empty(T, np.int32)
        child = np.empty(T, np.int32)
        flags = np.empty(T, np.uint8)
        coll = np.empty(T * 9, np.int32)
        il = np.empty(T * _lib.N_OFFSETS, np.int32)
        ordv = np.empty(fmm.N, np.int32)
        vp = lambda a: ctypes.c_void_p(a.ctypes.data)
        _lib.call("fmm_tree_export", plan, vp(xmin), vp(ymin), vp(bot), vp(top), vp(parent),
                  vp(child), vp(flags), vp(coll), vp(il), vp(ordv))
        coll = coll.reshape(T, 9)
        il = il.reshape(T, _lib.N_OFFSETS)
        off = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
        self.bbox = list(fmm.bbox)
        self.N = fmm.N
        self.ordv = ordv.astype(np.int64)
        self.levels = L
        self.Levels = []
        self._il = []
        grid49 = np.array([(a + 3) * 7 + (b + 3) for a in range(-3, 4) for b in range(-3, 4)
                           if not (abs(a) <= 1 and abs(b) <= 1)])
        for m in range(L):
            a, b = off[m], off[m + 1]
            lv = TreeLevel()
            lv.width = widths[m]
            lv.half_width = 0.5 * widths[m]
            lv.n_node = int(b - a)
            lv.xmin = xmin[a:b]
            lv.ymin = ymin[a:b]
            lv.xmid = lv.xmin + lv.half_width
            lv.ymid = lv.ymin + lv.half_width
            lv.bot_ind = bot[a:b].astype(np.int64)
            lv.top_ind = top[a:b].astype(np.int64)
            lv.ns = lv.top_ind - lv.bot_ind
            f = flags[a:b]
            lv.leaf = (f & 1) != 0
            lv.fake_leaf = (f & 2) != 0
            lv.Xlist = (f & 4) != 0
            ch = child[a:b].astype(np.int64)
            lv.children_ind = np.where(ch >= 0, ch - off[m + 1] if m + 1 <= L else ch, -1)
            par = parent[a:b].astype(np.int64)
            lv.parent_ind = np.where(par >= 0, par - (off[m - 1] if m > 0 else 0), -1)
            c = coll[a:b].astype(np.int64)
            lv.colleagues = np.where(c >= 0, c - a, -1)
            lv.compute_upwards = ((lv.leaf & ~lv.Xlist) | lv.fake_leaf) & (lv.ns > 0)
            lv.compute_downwards = (~lv.leaf | lv.Xlist) & ~lv.fake_leaf
            self.Levels.append(lv)
            rows = il[a:b]
            t, o = np.nonzero(rows >= 0)
            self._il.append(np.stack([t, grid49[o], rows[t, o].astype(np.int64) - a], axis=1)
                            if t.size else np.zeros((0, 3), np.int64))

    def interaction_triples(self, ind):
        """(target node, offset id (ox+3)*7+(oy+3), source node) of level ``ind``."""
        return self._il[ind]


class KI_FMM:
    """Kernel-independent FMM (KI_FMM, flexmm/flexmm2d/kifmm.py:122-144)."""

    _helper_cls = KI_Helper
    _max_nequiv = _lib.MAX_NEQUIV

    @staticmethod
    def _default_helper(kernel, nequiv):
        return default_helper(kernel, nequiv)

    def __init__(self, x, y, kernel_eval, Ncutoff=50, Nequiv=50, dtype=float, bbox=None,
                 helper=None, verbose=False, precision="fp64", **kernel_params):
        if dtype not in (float, np.float64):
            raise NotImplementedError("only real float64 charges are supported")
        # the points first: from pinned host memory their copies run while
        # the rest of the set-up is done on the host
        xd, _ = _device_f64(x)
        yd, _ = _device_f64(y)
        if Nequiv > self._max_nequiv:
            raise ValueError(f"Nequiv must be <= {self._max_nequiv}")
        if precision not in _lib.PRECISION:
            raise ValueError(f"precision must be one of {sorted(_lib.PRECISION)}")
        self.precision = precision
        _lib.load()
        self.kernel = resolve(kernel_eval, **kernel_params)
        if self.kernel.vector:
            raise ValueError(f"{self.kernel.name} is vector valued: its FMM is "
                             "flexmm_b200.stokes.FMM (kifmm2d/vector/stokes_fmm.py)")
        self.Ncutoff = int(Ncutoff)
        self.Nequiv = int(Nequiv)
        self.dtype = dtype
        self.verbose = verbose
        self.helper = helper if helper is not None else self._default_helper(self.kernel, self.Nequiv)
        if not isinstance(self.helper, self._helper_cls):
            raise TypeError(f"helper must be a flexmm_b200 {self._helper_cls.__name__}")
        self.helper.attach(self.kernel, self.Nequiv)
        if xd.numel() != yd.numel():
            raise ValueError("x and y differ in length")
        self.N = int(xd.numel())
        if bbox is None:
            bb = [xd.min().item(), xd.max().item(), yd.min().item(), yd.max().item()]
        else:
            bb = [float(v) for v in bbox]
        # a repeated bbox (a solver's every step) snaps and binds from a memo
        # on the helper: host time here delays the tree's first launch
        memo = self.helper.__dict__.setdefault("_ctor_memo", {})
        if len(memo) > 256:
            memo.clear()
        bkey = ("bbox", tuple(bb), len(self.helper.precomputations))
        snapped = memo.get(bkey)
        if snapped is None:
            snapped = memo[bkey] = tuple(self.helper.get_bbox(None, None, bb))
        self.bbox = list(snapped)
        st = time.time()
        plan = ctypes.c_void_p()
        bb_arr = (ctypes.c_double * 4)(*self.bbox)
        _lib.call("fmm_plan_create", self.helper.ops_set().handle, ctypes.c_void_p(xd.data_ptr()),
                  ctypes.c_void_p(yd.data_ptr()), self.N, self.Ncutoff, bb_arr, _stream(),
                  ctypes.byref(plan))
        self._plan = plan
        self._ops = self.helper.ops_set()   # keep the operator set alive with the plan
        _lib.call("fmm_plan_set_precision", plan, _lib.PRECISION[precision])
        self._x, self._y = xd, yd
        # the caller's own source objects: evaluating at them again reuses the
        # tree's sorted copy, as long as torch's version counters show them unchanged
        torch = _torch()
        self._src_in = ((x, y, x._version, y._version)
                        if isinstance(x, torch.Tensor) and isinstance(y, torch.Tensor) else None)
        nl = ctypes.c_int()
        widths = (ctypes.c_double * _lib.MAX_LEVELS)()
        # level count and widths only: the per-level node counts would wait for
        # the GPU (the tree's last kernels still run while the plan is set up)
        _lib.call("fmm_plan_info", plan, ctypes.byref(nl), widths, None)
        self._levels = nl.value
        self._widths = [widths[i] for i in range(nl.value)]
        if verbose:
            print("....Tree formed in:             {:0.1f}".format((time.time() - st) * 1000))
        # operators for every level width (KI_Helper.prepare, flexmm/flexmm2d/kifmm.py:67-82)
        ikey = ("ids", tuple(self._widths), id(self.helper.ops_set()))
        ids = memo.get(ikey)
        if ids is None:
            ids = memo[ikey] = (ctypes.c_int * nl.value)(*[self.helper.level_id(w) for w in self._widths])
        _lib.call("fmm_plan_bind_levels", plan, nl.value, ctypes.cast(ids, ctypes.c_void_p))
        self._tree = None
        self._expanded = False
        # named evaluators (kifmm2d FMM.__init__ registers 'potential_evaluation')
        self._evaluators = {"potential_evaluation": "potential"}
        # named upwardors (kifmm2d FMM.__init__ registers 'slp')
        self._upwardors = {"slp": "slp"}

    @property
    def _counts(self):
        """Nodes per level (waits for the tree's construction to finish)."""
        counts = (ctypes.c_int * _lib.MAX_LEVELS)()
        _lib.call("fmm_plan_info", self._plan, None, None, counts)
        return [counts[i] for i in range(self._levels)]

    @property
    def tree(self):
        if self._tree is None:
            self._tree = TreeView(self)
        return self._tree

    # device upwardors: the reference compiles a user's numba source function
    # (KAS(sx, sy, tx, ty, tau, extras)) into its S2M loop; here a function is
    # mapped by its name to the built-in device form of the same sum
    _UPWARDOR_KINDS = {"slp": "slp", "extra_kernel_app": "slp", "kernel_app": "slp",
                       "slp+dlp": "slp+dlp", "Laplace_Both_Eval": "slp+dlp"}

    def register_upwardor(self, KAS, name):
        """Name a source-to-multipole form (kifmm2d FMM.register_upwardor,
        flexmm/kifmm2d/scalar/fmm.py:174-176, helpers.py:155-173).  Built in:
        'slp' (charges) and 'slp+dlp' (charges and dipoles: the reference
        example's Laplace_Both_Eval, examples/pure_kifmm_laplace_dipoles.py:31-40,
        with tau = [charge, dipole strength] and extras = normals [nx, ny]).
        KAS is that function (matched by its name) or one of those names."""
        key = KAS if isinstance(KAS, str) else getattr(getattr(KAS, "py_func", KAS), "__name__", None)
        kind = self._UPWARDOR_KINDS.get(key)
        if kind is None:
            raise NotImplementedError(f"no device form of upwardor {key!r}; built in: "
                                      f"{sorted(self._UPWARDOR_KINDS)}")
        if kind == "slp+dlp" and self.kernel.kernel_id != 0:
            raise NotImplementedError("the double layer is built in for Laplace_Eval only")
        self._upwardors[name] = kind

    def build_expansions(self, tau, name=None, extras=None):
        """Charges in the caller's source order: [N], or [k, N] for k charge
        columns on one tree (FP64 form), whose evaluations then return [k, M].

        ``name`` selects a registered upwardor (kifmm2d's
        build_expansions(tau, name, extras), flexmm/kifmm2d/scalar/fmm.py:168-170):
        with an 'slp+dlp' upwardor tau is [2, N] (charge, dipole strength)
        and ``extras`` [2, N] the dipole normals, and every later evaluation
        includes both layers."""
        kind = "slp" if name is None else self._upwardors.get(name)
        if kind is None:
            raise KeyError(f"upwardor {name!r} is not registered; registered: {sorted(self._upwardors)}")
        if kind == "slp+dlp":
            return self._build_dipole(tau, extras)
        self._n_rhs = None
        if np.ndim(tau) == 2:
            torch = _torch()
            t = tau if isinstance(tau, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(tau, dtype=np.float64))
            td = t.to(device="cuda", dtype=torch.float64).contiguous()
            k, n = td.shape
            if n != self.N:
                raise ValueError(f"tau has {n} columns, expected {self.N}")
            if self.precision == "mixed":
                # mixed form: each evaluation runs every column through the
                # mixed passes on this tree (_evaluate_multi); nothing to build yet
                self._check_mixed_columns()
            else:
                _lib.call("fmm_build_expansions_multi", self._plan, ctypes.c_void_p(td.data_ptr()), k,
                          n, _stream())
            self._tau = td
            self._n_rhs = k
            self._expanded = True
            return
        td, _ = _device_f64_early(tau)
        if td.numel() != self.N:
            raise ValueError(f"tau has {td.numel()} entries, expected {self.N}")
        st = time.time()
        _lib.call("fmm_build_expansions", self._plan, ctypes.c_void_p(td.data_ptr()), _stream())
        self._tau = td   # kept alive until the stream has consumed it
        self._expanded = True
        if self.verbose:
            _torch().cuda.synchronize()
            print("....Time for expansions:        {:0.2f}".format(1000 * (time.time() - st)))

    def _build_dipole(self, tau, extras):
        if extras is None:
            raise ValueError("the 'slp+dlp' upwardor needs extras = [nx, ny] (dipole normals)")
        torch = _torch()
        dev = lambda a: (a if isinstance(a, torch.Tensor)
                         else torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)))
        t = dev(tau).to(device="cuda", dtype=torch.float64).contiguous()
        e = dev(extras).to(device="cuda", dtype=torch.float64).contiguous()
        if t.shape != (2, self.N) or e.shape != (2, self.N):
            raise ValueError(f"'slp+dlp' takes tau [2, {self.N}] and extras [2, {self.N}]")
        self._n_rhs = None
        p = lambda a: ctypes.c_void_p(a.data_ptr())
        _lib.call("fmm_build_expansions_dipole", self._plan, p(t[0]), p(t[1]), p(e[0]), p(e[1]),
                  _stream())
        self._tau, self._extras = t, e   # kept alive until the stream has consumed them
        self._expanded = True

    def drop_expansions(self):
        """Release the expansions, keep the tree; build_expansions forms them again."""
        _lib.call("fmm_plan_drop_expansions", self._plan)
        self._expanded = False
        self._tau = None

    def move_sources(self, x, y):
        """New source coordinates on the same (frozen) tree: every source keeps
        the leaf it was sorted into; expansions must be built again."""
        xd, _ = _device_f64(x)
        yd, _ = _device_f64(y)
        if xd.numel() != self.N or yd.numel() != self.N:
            raise ValueError(f"expected {self.N} source coordinates")
        _lib.call("fmm_plan_move_sources", self._plan, ctypes.c_void_p(xd.data_ptr()),
                  ctypes.c_void_p(yd.data_ptr()), _stream())
        self._x, self._y = xd, yd
        torch = _torch()
        self._src_in = ((x, y, x._version, y._version)
                        if isinstance(x, torch.Tensor) and isinstance(y, torch.Tensor) else None)
        self._expanded = False
        self._tau = None

    def register_evaluator(self, KAS1, KAS2, name, outputs):
        """Name an evaluator (kifmm2d FMM.register_evaluator, flexmm/kifmm2d/scalar/fmm.py:172-173).

        The reference compiles the user's pair of numba functions (L2T and
        P2P forms) into its loops.  Here the device evaluators are built in
        and the pair selects one by its output count: 1 output is the
        potential, 3 outputs are the potential and its gradient in the target
        position (u, du/dx, du/dy), as the reference's gradient example
        defines them (examples/pure_kifmm_laplace_gradient.py:32-55)."""
        if outputs == 1:
            self._evaluators[name] = "potential"
        elif outputs == 3:
            self._evaluators[name] = "gradient"
        else:
            raise NotImplementedError("built-in evaluators have 1 (potential) or 3 (gradient) outputs")

    def evaluate_to_points(self, x, y, name, check):
        """Evaluator `name` at (x, y) -> [outputs, M] (flexmm/kifmm2d/scalar/fmm.py:178-199);
        `check` skips sources that coincide with the target."""
        if name not in self._evaluators:
            raise KeyError(f"evaluator {name!r} is not registered; registered: {sorted(self._evaluators)}")
        eid, nout = _lib.EVALUATORS[self._evaluators[name]]
        torch = _torch()
        if check and self._own_sources(x, y):
            out = torch.empty((nout, self.N), dtype=torch.float64, device="cuda")
            _lib.call("fmm_evaluate_sources_outputs", self._plan, eid, 1,
                      ctypes.c_void_p(out.data_ptr()), self.N, _stream())
            return _as_kind(out, "cuda" if x.is_cuda else "cpu", (nout, self.N))
        xd, kind = _device_f64(x)
        yd, _ = _device_f64(y)
        if xd.numel() != yd.numel():
            raise ValueError("x and y differ in length")
        m = xd.numel()
        out = torch.empty((nout, m), dtype=torch.float64, device="cuda")
        _lib.call("fmm_evaluate_outputs", self._plan, eid, ctypes.c_void_p(xd.data_ptr()),
                  ctypes.c_void_p(yd.data_ptr()), m, 1 if check else 0,
                  ctypes.c_void_p(out.data_ptr()), m, _stream())
        return _as_kind(out, kind, (nout, m))

    def _check_mixed_columns(self):
        if self.kernel.kernel_id not in (0, 1):
            raise NotImplementedError("mixed charge columns: Laplace and modified Helmholtz only")

    def _evaluate_columns_mixed(self, x, y, check, k):
        """Mixed form, k charge columns: the columns' expansions are formed one
        after another on this tree and each column is evaluated right after
        its own, into row c of the [k, M] result."""
        torch = _torch()
        own = check and self._own_sources(x, y)
        if own:
            m, kind = self.N, ("cuda" if x.is_cuda else "cpu")
        else:
            xd, kind = _device_f64(x)
            yd, _ = _device_f64(y)
            m = xd.numel()
        out = torch.empty((k, m), dtype=torch.float64, device="cuda")
        for c in range(k):
            _lib.call("fmm_build_expansions", self._plan, ctypes.c_void_p(self._tau[c].data_ptr()),
                      _stream())
            row = ctypes.c_void_p(out[c].data_ptr())
            if own:
                _lib.call("fmm_evaluate_sources", self._plan, 1, row, _stream())
            else:
                _lib.call("fmm_evaluate", self._plan, ctypes.c_void_p(xd.data_ptr()),
                          ctypes.c_void_p(yd.data_ptr()), m, 1 if check else 0, row, _stream())
        return _as_kind(out, kind, (k, m))

    def _evaluate_multi(self, x, y, check):
        torch = _torch()
        k = self._n_rhs
        if self.precision == "mixed":
            return self._evaluate_columns_mixed(x, y, check, k)
        if check and self._own_sources(x, y):
            out = torch.empty((k, self.N), dtype=torch.float64, device="cuda")
            _lib.call("fmm_evaluate_sources_multi", self._plan, 1, ctypes.c_void_p(out.data_ptr()),
                      self.N, _stream())
            return _as_kind(out, "cuda" if x.is_cuda else "cpu", (k, self.N))
        xd, kind = _device_f64(x)
        yd, _ = _device_f64(y)
        m = xd.numel()
        out = torch.empty((k, m), dtype=torch.float64, device="cuda")
        _lib.call("fmm_evaluate_multi", self._plan, ctypes.c_void_p(xd.data_ptr()),
                  ctypes.c_void_p(yd.data_ptr()), m, 1 if check else 0,
                  ctypes.c_void_p(out.data_ptr()), m, _stream())
        return _as_kind(out, kind, (k, m))

    def _evaluate(self, x, y, check):
        if getattr(self, "_n_rhs", None):
            return self._evaluate_multi(x, y, check)
        torch = _torch()
        xd, kind = _device_f64(x)
        yd, _ = _device_f64(y)
        if xd.numel() != yd.numel():
            raise ValueError("x and y differ in length")
        out = torch.empty(xd.numel(), dtype=torch.float64, device="cuda")
        _lib.call("fmm_evaluate", self._plan, ctypes.c_void_p(xd.data_ptr()),
                  ctypes.c_void_p(yd.data_ptr()), xd.numel(), 1 if check else 0,
                  ctypes.c_void_p(out.data_ptr()), _stream())
        return _as_kind(out, kind, np.shape(x))

    def _own_sources(self, x, y):
        si = self._src_in
        return (si is not None and x is si[0] and y is si[1] and x._version == si[2]
                and y._version == si[3])

    def source_evaluation(self, x, y):
        """Potential at (x, y), skipping coincident sources (flexmm/flexmm2d/fmm.py:158-159).

        Called with the very tensors the FMM was built on (unchanged), the
        evaluation runs on the tree's sorted copy of them (fmm_evaluate_sources)
        instead of uploading, locating and sorting the points again."""
        if not self._own_sources(x, y) or getattr(self, "_n_rhs", None):
            return self._evaluate(x, y, True)
        torch = _torch()
        out = torch.empty(self.N, dtype=torch.float64, device="cuda")
        _lib.call("fmm_evaluate_sources", self._plan, 1, ctypes.c_void_p(out.data_ptr()), _stream())
        return _as_kind(out, "cuda" if x.is_cuda else "cpu", tuple(x.shape))

    def target_evaluation(self, x, y):
        """Potential at (x, y) (flexmm/flexmm2d/fmm.py:160-161)."""
        return self._evaluate(x, y, False)

    def status(self):
        """Wait for this object's GPU work and raise if a kernel reported a failure."""
        _lib.call("fmm_plan_status", self._plan)

    def direct_evaluation(self, x, y, check=False):
        """FP64 direct sum of this object's sources and charges at (x, y)
        (kernel_apply / kernel_apply_single_check, flexmm/flexmm2d/helpers.py:91-116)."""
        if not self._expanded:
            raise RuntimeError("build_expansions has not run")
        return direct_evaluation(self.kernel, self._x, self._y, self._tau, x, y, check)

    def __del__(self):
        try:
            if getattr(self, "_plan", None) is not None and _lib._LIB is not None:
                _lib._LIB.fmm_plan_destroy(self._plan)
        except Exception:
            pass
        self._plan = None


def direct_evaluation(kernel, sx, sy, tau, tx, ty, check=False, **kernel_params):
    """FP64 direct sum on the GPU: u(t) = sum_s K(s, t) tau_s, skipping
    coincident pairs when ``check`` (flexmm/flexmm2d/helpers.py:91-116)."""
    torch = _torch()
    k = resolve(kernel, **kernel_params)
    sxd, _ = _device_f64(sx)
    syd, _ = _device_f64(sy)
    td, _ = _device_f64(tau)
    txd, kind = _device_f64(tx)
    tyd, _ = _device_f64(ty)
    out = torch.empty(txd.numel(), dtype=torch.float64, device="cuda")
    params = (ctypes.c_double * 4)(*k.params)
    _lib.call("fmm_direct", k.kernel_id, params, ctypes.c_void_p(sxd.data_ptr()),
              ctypes.c_void_p(syd.data_ptr()), ctypes.c_void_p(td.data_ptr()), sxd.numel(),
              ctypes.c_void_p(txd.data_ptr()), ctypes.c_void_p(tyd.data_ptr()), txd.numel(),
              1 if check else 0, ctypes.c_void_p(out.data_ptr()), _stream())
    return _as_kind(out, kind, np.shape(tx))


def set_split_evaluation(mode=None):
    """Own-source evaluation split into a near-field kernel beside the level
    passes and a far-field kernel after them: True / False, or None for the
    default (on for both forms)."""
    _lib.load()
    _lib.call("fmm_set_split_evaluation", -1 if mode is None else int(bool(mode)))


def enable_timing(on=True):
    """Per-kernel CUDA-event timing inside the library (off by default)."""
    _lib.load()
    _lib.call("fmm_timing_enable", 1 if on else 0)


def read_timing():
    """{phase: (milliseconds, timed launches)} since the last read."""
    ms = (ctypes.c_double * _lib.N_PHASES)()
    n = (ctypes.c_int64 * _lib.N_PHASES)()
    _lib.call("fmm_timing_read", ms, n)
    return {name: (ms[i], n[i]) for i, name in enumerate(_lib.PHASES)}
