"""Differentiable FMM potential: a torch.autograd.Function whose backward is
the transposed FMM.

    u_i = sum_j K(s_j, t_i) tau_j          (forward: one FMM over the sources)

For a translation-invariant, symmetric kernel K(s, t) = f(t - s) = f(s - t)
and an upstream gradient r = dL/du:

* dL/dtau_j = sum_i r_i K(t_i, s_j) = phi(s_j), phi the field of charges r
  at the targets: the adjoint FMM (sources and targets exchanged);
* dL/ds_j   = tau_j grad phi(s_j): the adjoint FMM's gradient evaluator at
  the sources (grad_s f(t - s) = grad_x f(x - t) at x = s);
* dL/dt_i   = r_i grad u(t_i): the forward FMM's gradient evaluator at the
  targets.

The reference has no adjoint (its FMMs are forward only); this is the
differentiation form of the black-box and kernel-independent FMMs here.

Memory: the forward keeps the tree it built (its FMM plan) but not the
expansions -- they are released right after the forward evaluation and
formed again in the backward pass from the saved charges, when target
gradients are asked for.  The adjoint FMM builds its own tree over the
targets, forms the expansions of r, evaluates, and releases them.

``fmm_potential`` builds both trees per call.  ``FMMPotential`` builds them
once and keeps them frozen: later calls move the points inside the existing
trees (every point keeps its leaf), which is what a central-difference check
"with the tree frozen" differentiates, and what an optimisation loop over
slowly moving points wants.
"""
import torch

from .bbfmm import BB_FMM, BB_Helper
from .helpers import KI_Helper
from .kifmm import KI_FMM


_HELPERS = {}   # operator caches shared by every call with the same method, kernel and order


def _helper(method, kernel, order, kernel_params):
    key = (method, kernel if isinstance(kernel, str) else id(kernel), order,
           tuple(sorted(kernel_params.items())))
    if key not in _HELPERS:
        _HELPERS[key] = BB_Helper() if method == "bb" else KI_Helper()
    return _HELPERS[key]


def _make(method, kernel, ncut, neq, p, bbox, kernel_params):
    if method == "bb":
        helper = _helper(method, kernel, p, kernel_params)

        def make(x, y):
            return BB_FMM(x, y, kernel, ncut, p, bbox=bbox, helper=helper, **kernel_params)
    elif method == "kifmm":
        helper = _helper(method, kernel, neq, kernel_params)

        def make(x, y):
            return KI_FMM(x, y, kernel, ncut, neq, bbox=bbox, helper=helper, **kernel_params)
    else:
        raise ValueError("method must be 'bb' or 'kifmm'")
    return make


class _Trees:
    """The forward FMM (tree over the sources) and the adjoint FMM (tree over
    the targets) of one differentiable evaluation.  ``frozen``: built once,
    later coordinates are moved into them; otherwise built on first use."""

    def __init__(self, make, frozen=False):
        self.make = make
        self.frozen = frozen
        self.F = None
        self.A = None

    def _get(self, which, x, y):
        fm = getattr(self, which)
        if fm is None:
            fm = self.make(x, y)
            fm.register_evaluator(None, None, "gradient", 3)
            setattr(self, which, fm)
        elif self.frozen:
            fm.move_sources(x, y)
        return fm

    def forward_fmm(self, sx, sy):
        return self._get("F", sx, sy)

    def adjoint_fmm(self, tx, ty):
        return self._get("A", tx, ty)


class _FMMPotential(torch.autograd.Function):
    @staticmethod
    def forward(ctx, sx, sy, tau, tx, ty, trees):
        F = trees.forward_fmm(sx.detach(), sy.detach())
        F.build_expansions(tau.detach())
        u = F.target_evaluation(tx.detach(), ty.detach())
        F.drop_expansions()   # formed again in backward from the saved charges
        ctx.save_for_backward(sx, sy, tau, tx, ty)
        ctx.trees = trees
        return u

    @staticmethod
    def backward(ctx, gu):
        sx, sy, tau, tx, ty = ctx.saved_tensors
        trees = ctx.trees
        need = ctx.needs_input_grad
        g = [None] * 5
        gu = gu.detach().to(torch.float64).contiguous()
        if need[3] or need[4]:
            # the forward tree, its expansions recomputed
            F = trees.F
            if trees.frozen:
                F.move_sources(sx.detach(), sy.detach())
            F.build_expansions(tau.detach())
            G = F.evaluate_to_points(tx.detach(), ty.detach(), "gradient", False)
            F.drop_expansions()
            g[3] = gu * G[1] if need[3] else None
            g[4] = gu * G[2] if need[4] else None
        if need[0] or need[1] or need[2]:
            A = trees.adjoint_fmm(tx.detach(), ty.detach())
            A.build_expansions(gu)
            Gs = A.evaluate_to_points(sx.detach(), sy.detach(), "gradient", False)
            A.drop_expansions()
            g[2] = Gs[0] if need[2] else None
            g[0] = tau.detach() * Gs[1] if need[0] else None
            g[1] = tau.detach() * Gs[2] if need[1] else None
        if not trees.frozen:
            ctx.trees = None
        return g[0], g[1], g[2], g[3], g[4], None


def fmm_potential(sx, sy, tau, tx, ty, kernel="Laplace_Eval", method="bb", Ncutoff=64, Nequiv=32,
                  p=16, bbox=None, **kernel_params):
    """Differentiable u(t) = sum_j K(s_j, t) tau_j (CUDA float64 tensors);
    gradients for tau and both point sets through the transposed FMM.
    ``bbox`` must contain the sources and the targets (both trees use it)."""
    make = _make(method, kernel, Ncutoff, Nequiv, p, bbox, kernel_params)
    return _FMMPotential.apply(sx, sy, tau, tx, ty, _Trees(make))


class FMMPotential:
    """``fmm_potential`` on trees built once over (sx, sy) and (tx, ty) and then
    frozen: ``P(sx, sy, tau, tx, ty)`` moves the points inside those trees
    (each keeps its leaf) and evaluates differentiably.  Point counts must
    stay those of construction."""

    def __init__(self, sx, sy, tx, ty, kernel="Laplace_Eval", method="bb", Ncutoff=64, Nequiv=32,
                 p=16, bbox=None, **kernel_params):
        make = _make(method, kernel, Ncutoff, Nequiv, p, bbox, kernel_params)
        self.trees = _Trees(make, frozen=True)
        self.trees.forward_fmm(sx.detach(), sy.detach())
        self.trees.adjoint_fmm(tx.detach(), ty.detach())

    def __call__(self, sx, sy, tau, tx, ty):
        return _FMMPotential.apply(sx, sy, tau, tx, ty, self.trees)
