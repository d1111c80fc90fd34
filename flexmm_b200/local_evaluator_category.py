"""Near-field-only evaluation with categories
(flexmm/flexmm2d/local_evaluator_category.py): every source and target
carries an integer category, and a source adds nothing at a target of its
own category (so a point never sees itself, nor the other points of its own
body).  The tree and the sums run on the GPU, as in
``flexmm_b200.local_evaluator``; categories are int64."""
import numpy as np

from .local_evaluator import LocalHelper, _LocalCore, _host  # noqa: F401


class LocalEvaluator(_LocalCore):
    """``LocalEvaluator(x, y, cat, kernel_eval, min_distance, ncutoff=20,
    dtype=float, bbox=None, helper=None, verbose=False)``, ``load_tau(tau)``,
    ``target_evaluation(x, y, cat, out)`` (local_evaluator_category.py:91-138)."""

    def __init__(self, x, y, cat, kernel_eval, min_distance, ncutoff=20, dtype=float, bbox=None,
                 helper=None, verbose=False, **kernel_params):
        if dtype not in (float, np.float64):
            raise NotImplementedError("only real float64 densities are supported")
        self.verbose = verbose
        self._setup(x, y, kernel_eval, min_distance, ncutoff, bbox, helper, kernel_params)
        torch = __import__("torch")
        c = torch.as_tensor(_host(cat), dtype=torch.int64).reshape(-1)
        if c.numel() != self.N:
            raise ValueError("one category per source")
        self.cat = cat
        self._scat = c.cuda()

    def target_evaluation(self, x, y, cat, out=None):
        return self.evaluate_to_points(x, y, cat, "neighbor_potential_target_evaluation", out)

    def evaluate_to_points(self, x, y, cat, name, out=None):
        if name != "neighbor_potential_target_evaluation":
            raise KeyError(f"evaluator {name!r} is not registered")
        res, kind = self._near(x, y, False, tcat=cat)
        return self._into(out, res, kind)
