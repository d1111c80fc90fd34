"""Many independent Stokes problems at once: forward and charge adjoint.

The reference evaluates one Stokes FMM at a time
(flexmm/kifmm2d/vector/stokes_fmm.py:592-858).  ``StokesBatch`` holds one
FMM per problem, all sharing the per-width operators, and spreads them over
several CUDA streams: every call queues device work only (no host waits), so
the small problems of a batch overlap on the GPU.

Forward, for each problem's own sources (coincident points skipped):
``(u, v, p) = A f`` with the reference's Stokeslet (stokes_fmm.py:161-184):
u = (1/4pi) [(-log(r^2)/2 + dx^2/r^2) fx + (dx dy/r^2) fy], v likewise,
p = (1/2pi) (dx fx + dy fy) / r^2, (dx, dy) = target - source.

Charge adjoint: the velocity block of the Stokeslet is symmetric under
exchanging the two points and the two components, so its transpose is the
same velocity operator; the pressure row p_i = (1/2pi) sum_j (x_i - x_j) .
f_j / r^2 transposes to d f_j = (1/2pi) sum_i g_p,i (x_i - x_j) / r^2, the
target-position gradient of the Laplace potential -log(r^2)/(4pi) with
charges g_p.  So ``A^T (g_u, g_v, g_p)`` = Stokes velocity of (g_u, g_v) plus
the Laplace gradient of g_p, both at the sources.
"""
import ctypes

import numpy as np

from . import _lib
from .kifmm import KI_FMM, _torch
from .helpers import KI_Helper
from .stokes import FMM as StokesFMM


class StokesBatch:
    """``StokesBatch(problems, Nequiv=32, Ncutoff=64, n_streams=8)`` with
    ``problems`` a list of ``(x, y)`` source arrays; ``forward(forces)`` with
    ``forces`` a list of ``(fx, fy)`` returns a list of ``(u, v, p)``;
    ``adjoint(cotangents)`` with a list of ``(gu, gv, gp)`` returns a list of
    ``(dfx, dfy)``.  Results are CUDA tensors (call ``torch.cuda.synchronize``
    or read them, which waits, before using them on the host)."""

    def __init__(self, problems, Nequiv=32, Ncutoff=64, n_streams=8, adjoint=True,
                 precomputations=None):
        """``precomputations``: the operators of an earlier batch with the same
        Nequiv (``batch.precomputations``), so that widths it met are not
        formed again."""
        torch = _torch()
        self.Nequiv, self.Ncutoff = int(Nequiv), int(Ncutoff)
        self.streams = [torch.cuda.Stream() for _ in range(max(1, int(n_streams)))]
        self._pts, self._stokes, self._laplace = [], [], []
        pre = dict(precomputations) if precomputations else {}
        problems = list(problems)
        n = len(problems)
        # Trees: problem 0 first; its level widths fix the dyadic family every
        # later box snaps to (Stokes FMM adjust_bbox, stokes_fmm.py:608-637),
        # whatever deeper widths later problems add, so the other trees can be
        # built concurrently (each on its stream, from a pool of host threads:
        # the tree build's host waits then overlap) with their snapped boxes
        # computed up front.  Operators are bound afterwards, in problem order.
        def build(k, bbox, pre_k):
            x, y = problems[k]
            with torch.cuda.stream(self._stream(k)):
                xd = torch.as_tensor(np.asarray(x, dtype=np.float64)).cuda()
                yd = torch.as_tensor(np.asarray(y, dtype=np.float64)).cuda()
                return StokesFMM(xd, yd, self.Nequiv, self.Ncutoff, bbox,
                                 precomputations=pre_k if pre_k else None), xd, yd
        fmms = [None] * n
        if n:
            fmms[0] = build(0, None, pre)
            with torch.cuda.stream(self._stream(0)):
                fmms[0][0].precompute()
            pre = fmms[0][0].precomputations
        if n > 1:
            from concurrent.futures import ThreadPoolExecutor
            boxes = [None] + [[float(np.min(x)), float(np.max(x)), float(np.min(y)), float(np.max(y))]
                              for x, y in (map(np.asarray, problems[k]) for k in range(1, n))]
            with ThreadPoolExecutor(max_workers=len(self.streams)) as ex:
                for k, r in zip(range(1, n), ex.map(lambda k: build(k, boxes[k], pre), range(1, n))):
                    fmms[k] = r
            pre0 = pre   # the widths every later box was snapped to
            for k in range(1, n):
                F = fmms[k][0]
                F.input_precomputations = pre   # every width met so far: none formed twice
                with torch.cuda.stream(self._stream(k)):
                    F.precompute()
                pre = F.precomputations  # operators shared by width across problems
                # the operators this problem's box was snapped with (the same
                # problem built alone with them gets the same box and tree)
                F.input_precomputations = pre0
        helper = KI_Helper()
        for k in range(n):
            F, xd, yd = fmms[k]
            self._stokes.append(F)
            L = None
            if adjoint:
                with torch.cuda.stream(self._stream(k)):
                    L = KI_FMM(xd, yd, "Laplace_Eval", self.Ncutoff, self.Nequiv, helper=helper)
                L.register_evaluator(None, None, "gradient", 3)  # (u, du/dx, du/dy)
            self._laplace.append(L)
            self._pts.append((xd, yd))
        self.precomputations = pre
        torch.cuda.synchronize()

    def _stream(self, k):
        return self.streams[k % len(self.streams)]

    def __len__(self):
        return len(self._pts)

    def _own_stokes(self, F, n):
        torch = _torch()
        out = torch.empty((3, n), dtype=torch.float64, device="cuda")
        _lib.call("fmm_evaluate_sources_outputs", F._plan, _lib.EVALUATORS["stokes"][0], 1,
                  ctypes.c_void_p(out.data_ptr()), n,
                  ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
        return out

    def forward(self, forces):
        """(u, v, p) at every problem's sources for forces [(fx, fy), ...]."""
        torch = _torch()
        if len(forces) != len(self):
            raise ValueError(f"expected {len(self)} force pairs, got {len(forces)}")
        self._enter()
        outs = []
        for k, (F, (fx, fy)) in enumerate(zip(self._stokes, forces)):
            s = self._stream(k)
            with torch.cuda.stream(s):
                F.build_expansions(_device(fx, s), _device(fy, s))
                o = self._own_stokes(F, F.N)
                outs.append((o[0], o[1], o[2]))
        self._join(outs)
        return outs

    def adjoint(self, cotangents):
        """(dfx, dfy) = A^T (gu, gv, gp) for every problem."""
        torch = _torch()
        if any(L is None for L in self._laplace):
            raise RuntimeError("built with adjoint=False")
        if len(cotangents) != len(self):
            raise ValueError(f"expected {len(self)} cotangent triples, got {len(cotangents)}")
        self._enter()
        outs = []
        for k, (F, L, (gu, gv, gp), (xd, yd)) in enumerate(
                zip(self._stokes, self._laplace, cotangents, self._pts)):
            s = self._stream(k)
            with torch.cuda.stream(s):
                F.build_expansions(_device(gu, s), _device(gv, s))
                vel = self._own_stokes(F, F.N)
                L.build_expansions(_device(gp, s))
                grad = L.evaluate_to_points(xd, yd, "gradient", True)
                outs.append((vel[0] + grad[1], vel[1] + grad[2]))
        self._join(outs)
        return outs

    def _enter(self):
        """Every batch stream waits for the caller's stream, so inputs the
        caller produced on the GPU just before the call are complete when the
        batch streams read them."""
        torch = _torch()
        cur = torch.cuda.current_stream()
        for s in self.streams:
            s.wait_stream(cur)

    def _join(self, outs):
        """The caller's stream waits for every batch stream, and the results
        (made on the batch streams) are marked as used on it."""
        torch = _torch()
        cur = torch.cuda.current_stream()
        for s in self.streams:
            cur.wait_stream(s)
        for tup in outs:
            for t in tup:
                t.record_stream(cur)

    def graph(self, kind="forward"):
        """A CUDA graph of one batch call (kind "forward" or "adjoint") over
        static input tensors: ``g.replay(inputs)`` copies the inputs into the
        graph's buffers, launches the whole batch -- every problem's S2M,
        level passes and evaluation on its stream -- as ONE graph launch, and
        returns the outputs (tensors owned by the graph, overwritten by the
        next replay).  The trees and operators stay those of this batch;
        capture runs one warm-up call first so that every plan's expansion
        buffers exist before capture (memory allocated inside the graph is
        only its per-call scratch)."""
        return _BatchGraph(self, kind)

    def status(self):
        for F in self._stokes:
            F.status()
        for L in self._laplace:
            if L is not None:
                L.status()


def _device(a, stream):
    """A contiguous float64 CUDA tensor of ``a`` for use on ``stream`` (the
    current stream inside the caller's ``torch.cuda.stream`` block).  A CUDA
    tensor the caller passed in is marked as used on that stream, so the
    caching allocator does not hand its memory out again before the batch
    stream has read it, even if the caller drops it right after the call."""
    torch = _torch()
    if isinstance(a, torch.Tensor):
        t = a.to(device="cuda", dtype=torch.float64).contiguous()
        if t.is_cuda and a.is_cuda and stream is not None:
            t.record_stream(stream)
        return t
    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64)).cuda()


class _BatchGraph:
    def __init__(self, batch, kind):
        torch = _torch()
        if kind not in ("forward", "adjoint"):
            raise ValueError("kind must be 'forward' or 'adjoint'")
        self.batch, self.kind = batch, kind
        width = 2 if kind == "forward" else 3
        self.inputs = [tuple(torch.zeros(int(xd.numel()), dtype=torch.float64, device="cuda")
                             for _ in range(width)) for xd, _ in batch._pts]
        fn = batch.forward if kind == "forward" else batch.adjoint
        side = torch.cuda.Stream()
        side.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(side):
            fn(self.inputs)          # warm-up: plan buffers, side streams, kernel attributes
        torch.cuda.current_stream().wait_stream(side)
        torch.cuda.synchronize()
        self.g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.g):
            self.outputs = fn(self.inputs)
        torch.cuda.synchronize()

    def replay(self, inputs=None):
        """Copy ``inputs`` (same structure as the batch call's) into the graph's
        buffers (None: keep the current ones), launch the graph, return the
        outputs."""
        if inputs is not None:
            if len(inputs) != len(self.inputs):
                raise ValueError(f"expected {len(self.inputs)} problems")
            for dst, src in zip(self.inputs, inputs):
                for d, v in zip(dst, src):
                    d.copy_(_device(v, None) if not hasattr(v, "is_cuda") else v, non_blocking=True)
        self.g.replay()
        return self.outputs
