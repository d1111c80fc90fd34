"""Periodic near-field evaluation with categories
(flexmm/flexmm2d/periodic_local_evaluator_category.py): sources live in the
periodic cell ``bounds``; every source within ``min_distance`` of a side
gets the image shifted by the cell width across that side (and a corner
source the images across both sides and the diagonal), and the category
evaluator runs on sources plus images over the cell grown by
``min_distance``.  Targets are shifted into the cell first.  Assumes
``min_distance`` below the cell size, as the reference does."""
import numpy as np

from .local_evaluator import _host
from .local_evaluator_category import LocalEvaluator


def shift_to_interval(v, interval):
    """Periodically shift values into [interval[0], interval[1])."""
    r = interval[1] - interval[0]
    return (np.asarray(v, dtype=np.float64) - interval[0]) % r + interval[0]


def periodic_images(x, y, c, bounds, min_distance):
    """Sources plus their images: (x, y, c, index of the original source).
    A source closer than min_distance to the left side is repeated shifted
    by +width, to the right side by -width, likewise in y; near a corner
    every nonzero combination of its x and y shifts is added (the image set
    of the reference's append(), periodic_local_evaluator_category.py:11-112)."""
    x, y, c = (np.asarray(v) for v in (x, y, c))
    xr, yr = bounds[1] - bounds[0], bounds[3] - bounds[2]
    sx = np.where(x < bounds[0] + min_distance, xr, np.where(x > bounds[1] - min_distance, -xr, 0.0))
    sy = np.where(y < bounds[2] + min_distance, yr, np.where(y > bounds[3] - min_distance, -yr, 0.0))
    idx = [np.arange(x.size)]
    xs, ys = [x], [y]
    for ax, ay in ((1, 0), (0, 1), (1, 1)):
        sel = np.flatnonzero(((sx != 0) | (ax == 0)) & ((sy != 0) | (ay == 0)))
        idx.append(sel)
        xs.append(x[sel] + ax * sx[sel])
        ys.append(y[sel] + ay * sy[sel])
    i = np.concatenate(idx)
    return np.concatenate(xs), np.concatenate(ys), c[i], i


class PeriodicLocalEvaluator:
    """``PeriodicLocalEvaluator(x, y, cat, kernel_eval, min_distance, bounds,
    ncutoff=20, dtype=float, helper=None, verbose=False)``, ``load_tau(tau)``,
    ``target_evaluation(x, y, cat, out)``."""

    def __init__(self, x, y, cat, kernel_eval, min_distance, bounds, ncutoff=20, dtype=float,
                 helper=None, verbose=False, **kernel_params):
        self.bounds = [float(b) for b in bounds]
        self.min_distance = float(min_distance)
        self.x = shift_to_interval(_host(x), self.bounds[0:2])
        self.y = shift_to_interval(_host(y), self.bounds[2:4])
        self.cat = np.asarray(_host(cat))
        md = self.min_distance
        self.bbox = [self.bounds[0] - md, self.bounds[1] + md, self.bounds[2] - md, self.bounds[3] + md]
        self.append_x, self.append_y, self.append_cat, self.append_ind = periodic_images(
            self.x, self.y, self.cat, self.bounds, md)
        self.LocalEvaluator = LocalEvaluator(self.append_x, self.append_y, self.append_cat,
                                             kernel_eval, md, ncutoff, dtype, self.bbox, helper,
                                             verbose, **kernel_params)

    def load_tau(self, tau):
        self.LocalEvaluator.load_tau(np.asarray(_host(tau))[self.append_ind])

    def target_evaluation(self, x, y, cat, out=None):
        x = shift_to_interval(_host(x), self.bounds[0:2])
        y = shift_to_interval(_host(y), self.bounds[2:4])
        return self.LocalEvaluator.evaluate_to_points(x, y, cat, "neighbor_potential_target_evaluation",
                                                      out)
