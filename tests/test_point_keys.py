"""The point-key rule of the tree build, restated in numpy (host only).

The device computes a point's 29 quadrant digits from the fixed-point cell
index q = (p - x0) 2^29 / w0 wherever q is farther than
margin = 2^-14 max(1, X / w0) from every integer (X the largest coordinate
of the box), and by the reference's FP64 descent (xmid = xmin + w/2, child
xmin = xmid - w/2 or xmid, strict '>'; flexmm/tree.py:127-189, 301-307)
elsewhere.  Both must give the same digits; here the rule is checked against
the descent itself on points placed on and one ulp beside the descent's
midpoints, in boxes away from the origin with non-dyadic widths.
"""
import numpy as np

MAXD = 29


def descent_digits(p, x0, w0):
    out = np.empty(p.size, dtype=np.int64)
    for i, v in enumerate(p):
        xmin, w, q = x0, w0, 0
        for _ in range(MAXD):
            hw = 0.5 * w
            xm = xmin + hw
            h = 1 if v > xm else 0
            q = 2 * q + h
            xmin = xm if h else xm - hw
            w = hw
        out[i] = q
    return out


def rule_digits(p, x0, w0, y0=None):
    big = max(abs(x0), abs(x0 + w0)) if y0 is None else max(abs(x0), abs(x0 + w0), abs(y0), abs(y0 + w0))
    margin = 2.0 ** -14 * max(1.0, big / w0)
    q = (p - x0) * (2.0 ** MAXD / w0)
    clear = np.abs(q - np.rint(q)) > margin
    fixed = np.clip(np.floor(q), 0, 2 ** MAXD - 1).astype(np.int64)
    out = descent_digits(p, x0, w0)
    return np.where(clear, fixed, out), clear


def _lines(p, x0, w0, levels):
    out, xmin, w = [], x0, w0
    for _ in range(levels):
        hw = 0.5 * w
        xm = xmin + hw
        out.append(xm)
        xmin = xm if p > xm else xm - hw
        w = hw
    return out


def test_fixed_point_rule_equals_descent():
    rng = np.random.default_rng(5)
    boxes = [(-1.0, 2.0), (1000.3, 0.9), (-3.7, 0.9), (0.1, 1e-3), (-2e5, 3.3)]
    for x0, w0 in boxes:
        pts = list(x0 + w0 * rng.random(400))
        for v in pts[:40]:  # midpoints of the descent and one ulp either side
            for m in _lines(v, x0, w0, MAXD):
                pts += [m, np.nextafter(m, -np.inf), np.nextafter(m, np.inf)]
        pts += [x0 - 0.1 * w0, x0, x0 + w0, x0 + 1.1 * w0]  # edges and outside
        p = np.array(pts)
        got, clear = rule_digits(p, x0, w0)
        np.testing.assert_array_equal(got, descent_digits(p, x0, w0))
        # near the origin (coordinates within a few widths) the fixed-point
        # path covers almost every point; far from it the margin grows with
        # |x| / w and more points take the descent (same digits, slower)
        if max(abs(x0), abs(x0 + w0)) / w0 <= 4:
            assert clear[:400].mean() > 0.99


def test_margin_covers_the_midpoint_rounding():
    """The descent's midpoints differ from the exact lines x0 + k w0 / 2^l by
    accumulated FP64 rounding; it stays far inside the margin (in q units)."""
    rng = np.random.default_rng(6)
    for x0, w0 in [(1000.3, 0.9), (-2e5, 3.3), (0.1, 1e-3)]:
        margin = 2.0 ** -14 * max(1.0, max(abs(x0), abs(x0 + w0)) / w0)
        worst = 0.0
        for v in x0 + w0 * rng.random(50):
            for lvl, m in enumerate(_lines(v, x0, w0, MAXD)):
                q = (m - x0) * (2.0 ** MAXD / w0)  # an integer for the exact line
                worst = max(worst, abs(q - np.rint(q)))
        assert worst < margin / 4, (x0, w0, worst, margin)
