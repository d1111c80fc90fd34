"""CPU oracle: numpy restatement of the reference KIFMM driver.

TEST INFRASTRUCTURE ONLY (see ``oracle/tree.py``).  Follows
flexmm/flexmm2d/kifmm.py (operators, S2M, C2E by LU, L2T),
flexmm/flexmm2d/fmm.py (upward / downward passes, evaluation) and
flexmm/flexmm2d/helpers.py (bbox snapping, M2L SVD compression, P2P),
with the same operator formulas and the same LU-based check-to-equivalent
solve, so that its results can be pinned to the reference's own outputs.
"""
import numpy as np
import scipy.linalg

from .tree import Tree

SVD_TOL = 1e-14   # flexmm/flexmm2d/helpers.py:197


def kernel_form(kernel, sx, sy, tx, ty):
    """out[j, i] = K(s_i, t_j) (kernel_form, flexmm/flexmm2d/helpers.py:127-151)."""
    return kernel(sx[None, :], sy[None, :], tx[:, None], ty[:, None])


def level_surfaces(width, theta):
    """Equivalent (small) and check (large) circles, flexmm/flexmm2d/kifmm.py:158-168."""
    dd = 0.0
    r1 = 0.5 * width * (np.sqrt(2) + dd)
    r2 = 0.5 * width * (4 - np.sqrt(2) - 2 * dd)
    return r1 * np.cos(theta), r1 * np.sin(theta), r2 * np.cos(theta), r2 * np.sin(theta)


class M2LOperator:
    """Dense, SVD-truncated or null M2L (M2L_Evaluator, flexmm/flexmm2d/helpers.py:5-33)."""

    def __init__(self, m2l, tol=SVD_TOL):
        self.m2l = m2l
        U, S, VT = np.linalg.svd(m2l)
        keep = np.flatnonzero(S > tol)
        self.kind = "null"
        if keep.size:
            r = keep[-1] + 1
            if 2 * r < m2l.shape[0]:
                self.kind = "svd"
                self.M2 = U[:, :r].copy()
                self.M1 = VT[:r] * S[:r, None]
                self.rank = r
            else:
                self.kind = "dense"

    def apply(self, mult_T):
        """Return M2L . mult_T for mult_T of shape [Neq, n]."""
        if self.kind == "dense":
            return self.m2l @ mult_T
        if self.kind == "svd":
            return self.M2 @ (self.M1 @ mult_T)
        return np.zeros_like(mult_T)


class Precomputation:
    """Per-width operators (KI_Precomputation, flexmm/flexmm2d/kifmm.py:13-62)."""

    def __init__(self, width, nequiv, kernel):
        self.width = width
        theta = np.linspace(0, 2 * np.pi, nequiv, endpoint=False)
        sx, sy, lx, ly = level_surfaces(width, theta)
        s2l = kernel_form(kernel, sx, sy, lx, ly)
        self.S2L_LU = scipy.linalg.lu_factor(s2l.copy(), check_finite=False)
        self.L2S_LU = scipy.linalg.lu_factor(s2l.copy(), check_finite=False)
        ssx, ssy, _, _ = level_surfaces(0.5 * width, theta)
        q = 0.25 * width
        cex = np.concatenate([ssx - q, ssx - q, ssx + q, ssx + q])
        cey = np.concatenate([ssy - q, ssy + q, ssy - q, ssy + q])
        self.M2MC = kernel_form(kernel, cex, cey, lx, ly)
        self.L2LC = self.M2MC.T
        self.M2LF = {}
        for ix in range(7):
            for iy in range(7):
                if abs(ix - 3) <= 1 and abs(iy - 3) <= 1:
                    continue
                m = kernel_form(kernel, sx + (ix - 3) * width, sy + (iy - 3) * width, sx, sy)
                self.M2LF[(ix, iy)] = M2LOperator(m)
        self.small_x, self.small_y, self.large_x, self.large_y = sx, sy, lx, ly


def snap_bbox(px, py, bbox, known_widths):
    """Square (and optionally width-snapped) bbox, flexmm/flexmm2d/helpers.py:52-72."""
    if bbox is None:
        bbox = [np.min(px), np.max(px), np.min(py), np.max(py)]
    if len(known_widths) > 0:
        small = np.min(known_widths)
        bw = max(bbox[1] - bbox[0], bbox[3] - bbox[2])
        width = 2 ** np.ceil(np.log2(bw / small)) * small
    else:
        width = max(bbox[1] - bbox[0], bbox[3] - bbox[2])
    cx = (bbox[1] + bbox[0]) / 2
    cy = (bbox[3] + bbox[2]) / 2
    return [cx - width / 2, cx + width / 2, cy - width / 2, cy + width / 2]


def _ranges_to_index(bots, tops):
    lens = tops - bots
    tot = int(lens.sum())
    seg = np.repeat(np.arange(bots.size), lens)
    off = np.arange(tot) - np.repeat(np.cumsum(lens) - lens, lens)
    return seg, np.repeat(bots, lens) + off


class KIFMM:
    """Oracle for KI_FMM (flexmm/flexmm2d/kifmm.py:122-144, fmm.py:32-176).

    ``kernel(sx, sy, tx, ty)`` is a vectorised numpy evaluator of the same
    scalar kernel the reference compiles with numba.  ``cache`` maps
    round(width, 12) to a Precomputation, like FloatDict
    (flexmm/flexmm2d/float_dict.py:23-24).
    """

    def __init__(self, x, y, kernel, Ncutoff=50, Nequiv=50, bbox=None, cache=None):
        self.kernel = kernel
        self.Nequiv = Nequiv
        self.cache = {} if cache is None else cache
        self.bbox = snap_bbox(x, y, bbox, np.array(list(self.cache.keys()), dtype=float))
        self.tree = Tree(x, y, Ncutoff, self.bbox)
        self.prec = []
        for lv in self.tree.Levels:
            key = round(lv.width, 12)
            if key not in self.cache:
                self.cache[key] = Precomputation(lv.width, Nequiv, kernel)
            self.prec.append(self.cache[key])

    # -- source to check surface, flexmm/flexmm2d/kifmm.py:96-105
    def _s2m(self, lv, prec, tau_o, pM, chunk=1 << 21):
        t = self.tree
        nodes = np.flatnonzero(lv.compute_upwards & (lv.this_density_ind >= 0))
        if nodes.size == 0:
            return
        seg, src = _ranges_to_index(lv.bot_ind[nodes], lv.top_ind[nodes])
        n_eq = self.Nequiv
        step = max(1, chunk // n_eq)
        acc = np.zeros((nodes.size, n_eq))
        for a in range(0, src.size, step):
            s = src[a:a + step]
            g = seg[a:a + step]
            dx = t.x[s] - lv.xmid[nodes[g]]
            dy = t.y[s] - lv.ymid[nodes[g]]
            k = self.kernel(dx[:, None], dy[:, None], prec.large_x[None, :], prec.large_y[None, :])
            np.add.at(acc, g, k * tau_o[s][:, None])
        pM[lv.this_density_ind[nodes]] = acc

    def build_expansions(self, tau):
        t = self.tree
        L = t.levels
        n_eq = self.Nequiv
        tau = np.asarray(tau, dtype=np.float64)
        tau_o = tau[t.ordv]
        self.tau_ordered = tau_o
        mult = [None] * L
        resh = [None] * L
        # upward pass, flexmm/flexmm2d/fmm.py:67-107
        for ind in reversed(range(2, L)):
            lv = t.Levels[ind]
            prec = self.prec[ind]
            pM = np.zeros((lv.n_allocate_density, n_eq))
            if ind != L - 1:
                ch = t.Levels[ind + 1]
                temp = (prec.M2MC @ resh[ind + 1].T).T
                g = np.flatnonzero(ch.parent_density_ind >= 0)
                pM[lv.this_density_ind[ch.short_parent_ind[g]]] = temp[ch.parent_density_ind[g]]
            self._s2m(lv, prec, tau_o, pM)
            mult[ind] = scipy.linalg.lu_solve(prec.S2L_LU, pM.T, check_finite=False).T.copy()
            resh[ind] = mult[ind].reshape(lv.n_allocate_density // 4, 4 * n_eq)
        self.multipoles = mult
        # downward pass, flexmm/flexmm2d/fmm.py:108-149
        loc = [None] * L
        ple = [None] * L
        for ind in range(min(L, 2)):
            loc[ind] = np.zeros((t.Levels[ind].n_node, n_eq))
        if L > 2:
            ple[2] = np.zeros((t.Levels[2].n_node, n_eq))
        for ind in range(2, L):
            lv = t.Levels[ind]
            prec = self.prec[ind]
            dil = t.interaction_lists[ind]
            for (ix, iy), op in prec.M2LF.items():
                Y = op.apply(mult[ind].T).T
                sel = np.flatnonzero(dil[ix, iy] >= 0)
                ple[ind][sel] += Y[dil[ix, iy, sel]]
            loc[ind] = scipy.linalg.lu_solve(prec.L2S_LU, ple[ind].T, check_finite=False).T.copy()
            if ind < L - 1:
                doit = lv.compute_downwards
                p = (prec.L2LC @ loc[ind][doit].T).T
                order = np.argsort(lv.children_ind[doit], kind="stable")
                ple[ind + 1] = p[order].reshape(t.Levels[ind + 1].n_node, n_eq)
        self.Local_Expansions = loc

    def _evaluate(self, x, y, check, chunk=1 << 22):
        t = self.tree
        x = np.ascontiguousarray(x, dtype=np.float64).ravel()
        y = np.ascontiguousarray(y, dtype=np.float64).ravel()
        inds, locs = t.locate_points(x, y)
        pot = np.zeros(x.size)
        # L2T, flexmm/flexmm2d/kifmm.py:106-120
        for ind in np.unique(inds):
            sel = np.flatnonzero(inds == ind)
            lv = t.Levels[ind]
            prec = self.prec[ind]
            lo = locs[sel]
            dx = x[sel] - lv.xmid[lo]
            dy = y[sel] - lv.ymid[lo]
            k = self.kernel(prec.large_x[None, :], prec.large_y[None, :], dx[:, None], dy[:, None])
            pot[sel] = np.einsum("ij,ij->i", k, self.Local_Expansions[ind][lo])
        # P2P over colleagues, flexmm/flexmm2d/helpers.py:152-194
        order = np.lexsort((locs, inds))
        for ind in np.unique(inds):
            lv = t.Levels[ind]
            sel = order[inds[order] == ind]
            col = lv.colleagues[locs[sel]]                      # n x 9
            ok = col >= 0
            c = np.where(ok, col, 0)
            b = np.where(ok, lv.bot_ind[c], 0)
            e = np.where(ok, lv.top_ind[c], 0)
            tgt = np.repeat(sel, 9)
            seg, src = _ranges_to_index(b.ravel(), e.ravel())
            tg = tgt[seg]
            for a in range(0, src.size, chunk):
                s = src[a:a + chunk]
                ti = tg[a:a + chunk]
                dxs = x[ti] - t.x[s]
                dys = y[ti] - t.y[s]
                val = self.kernel(t.x[s], t.y[s], x[ti], y[ti]) * self.tau_ordered[s]
                if check:
                    val = np.where((dxs == 0) & (dys == 0), 0.0, val)
                pot += np.bincount(ti, weights=val, minlength=x.size)
        return pot

    def source_evaluation(self, x, y):
        with np.errstate(divide="ignore", invalid="ignore"):
            return self._evaluate(x, y, True)

    def target_evaluation(self, x, y):
        with np.errstate(divide="ignore", invalid="ignore"):
            return self._evaluate(x, y, False)
