"""CPU oracle: a numpy restatement of the reference quadtree.

TEST INFRASTRUCTURE ONLY.  Nothing in the product path (``flexmm_b200``)
imports this module; it is used by ``tests/``, ``__graft_entry__.smoke()``
and the ``cpu_baseline`` leg of ``bench.py`` as the checker.

It follows the reference's own algorithm step by step (level-by-level splits
of nodes holding more than ``ppl`` points, the 2:1 level-restriction fixpoint,
the X-list split into fake leaves, post-processing and 7x7 interaction lists)
so that it can be pinned against outputs of the reference itself
(``tests/golden``).  The GPU tree in ``flexmm_b200`` is built by a different
algorithm (point keys, radix sort, bottom-up balance closure) and is compared
with this one canonically (box coordinates, flags, leaf point sets, colleague
sets and interaction lists), independent of node numbering.

Reference citations are ``flexmm/tree.py:<line>``.
"""
import numpy as np

# flexmm/tree.py:11 -- below this many nodes a level tags colleagues directly
TREE_SEARCH_CROSSOVER = 100


class Level:
    """Nodes of one tree level (flexmm/tree.py:275-360)."""

    def __init__(self, xmin, ymin, width, bot, top, parent):
        self.xmin = np.asarray(xmin, dtype=np.float64)
        self.ymin = np.asarray(ymin, dtype=np.float64)
        self.width = width
        self.half_width = 0.5 * width
        self.bot_ind = np.asarray(bot, dtype=np.int64)
        self.top_ind = np.asarray(top, dtype=np.int64)
        self.parent_ind = np.asarray(parent, dtype=np.int64)
        n = self.xmin.shape[0]
        self.leaf = np.ones(n, dtype=bool)
        self.fake_leaf = np.zeros(n, dtype=bool)
        self.children_ind = -np.ones(n, dtype=np.int64)
        self._derive()

    def _derive(self):
        # flexmm/tree.py:301-308
        self.ns = self.top_ind - self.bot_ind
        self.xmid = self.xmin + self.half_width
        self.ymid = self.ymin + self.half_width
        self.n_node = self.xmin.shape[0]
        self.short_parent_ind = self.parent_ind[::4]

    def append(self, xmin, ymin, bot, top, parent, fake):
        """Append a batch of children (flexmm/tree.py:344-355)."""
        k = xmin.shape[0]
        self.xmin = np.concatenate([self.xmin, xmin])
        self.ymin = np.concatenate([self.ymin, ymin])
        self.bot_ind = np.concatenate([self.bot_ind, bot])
        self.top_ind = np.concatenate([self.top_ind, top])
        self.parent_ind = np.concatenate([self.parent_ind, parent])
        self.leaf = np.concatenate([self.leaf, np.full(k, not fake)])
        self.fake_leaf = np.concatenate([self.fake_leaf, np.full(k, fake)])
        self.children_ind = np.concatenate([self.children_ind, -np.ones(k, np.int64)])
        self._derive()


def _split(level, mask, x, y, ordv, child_start, xlist):
    """Split every node of ``level`` flagged in ``mask`` into 4 children.

    Restates divide_and_reorder (flexmm/tree.py:127-189): the points of each
    split node are regrouped by child class 2*(x > xmid) + (y > ymid)
    (classify, flexmm/tree.py:13-36).  The reference partitions in place and
    unstably; this regroups stably, which changes only the order of points
    inside a leaf, never which leaf a point is in.
    Returns (xmin, ymin, bot, top, parent) of the new children.
    """
    idx = np.flatnonzero(mask)
    k = idx.size
    hw = level.half_width
    bots = level.bot_ind[idx]
    tops = level.top_ind[idx]
    lens = tops - bots
    counts = np.zeros((k, 4), dtype=np.int64)
    if lens.sum() > 0:
        seg = np.repeat(np.arange(k), lens)
        starts = np.repeat(np.cumsum(lens) - lens, lens)
        pos = np.repeat(bots, lens) + (np.arange(lens.sum()) - starts)
        cls = 2 * (x[pos] > level.xmid[idx][seg]).astype(np.int64) \
            + (y[pos] > level.ymid[idx][seg]).astype(np.int64)
        order = np.lexsort((cls, seg))
        src = pos[order]
        x[pos] = x[src]
        y[pos] = y[src]
        ordv[pos] = ordv[src]
        np.add.at(counts, (seg, cls), 1)
    cum = np.zeros((k, 5), dtype=np.int64)
    cum[:, 1:] = np.cumsum(counts, axis=1)
    xm = level.xmid[idx]
    ym = level.ymid[idx]
    # child order (LL, LU, RL, RU) = classes 0..3, flexmm/tree.py:169-184
    nxmin = np.stack([xm - hw, xm - hw, xm, xm], axis=1).ravel()
    nymin = np.stack([ym - hw, ym, ym - hw, ym], axis=1).ravel()
    nbot = (bots[:, None] + cum[:, :4]).ravel()
    ntop = (bots[:, None] + cum[:, 1:]).ravel()
    ntop[3::4] = tops
    nparent = np.repeat(idx, 4)
    if not xlist:
        level.leaf[idx] = False
    level.children_ind[idx] = child_start + 4 * np.arange(k)
    return nxmin, nymin, nbot, ntop, nparent


def _pack_rows(cand, keep, width=9):
    """Keep the flagged entries of each row, in order, padded with -1."""
    order = np.argsort(~keep, axis=1, kind="stable")[:, :width]
    vals = np.take_along_axis(cand, order, axis=1)
    ok = np.take_along_axis(keep, order, axis=1)
    vals = np.where(ok, vals, -1)
    if vals.shape[1] < width:
        vals = np.concatenate([vals, -np.ones((vals.shape[0], width - vals.shape[1]), np.int64)], axis=1)
    return vals


def _tag_colleagues(level, ancestor):
    """Same-level nodes closer than 1.5 widths, self included, at most 9.

    Small levels compare all pairs (numba_tag_colleagues,
    flexmm/tree.py:222-234); larger ones look among the children of the
    parent's colleagues that have children (numba_loop_colleagues,
    flexmm/tree.py:236-256, called with children_ind < 0 as the leaf test,
    flexmm/tree.py:329-335).
    """
    n = level.n_node
    dist2 = (1.5 * level.width) ** 2
    if n < TREE_SEARCH_CROSSOVER or ancestor is None:
        dx = level.xmid[:, None] - level.xmid[None, :]
        dy = level.ymid[:, None] - level.ymid[None, :]
        keep = dx * dx + dy * dy < dist2
        cand = np.broadcast_to(np.arange(n), (n, n))
        level.colleagues = _pack_rows(np.ascontiguousarray(cand), keep)
        return
    pc = ancestor.colleagues[level.parent_ind]               # n x 9
    has = pc >= 0
    pch = np.where(has, ancestor.children_ind[np.where(has, pc, 0)], -1)
    has &= pch >= 0
    cand = (np.where(has, pch, 0)[:, :, None] + np.arange(4)[None, None, :]).reshape(n, 36)
    valid = np.repeat(has, 4, axis=1)
    dx = level.xmid[:, None] - level.xmid[cand]
    dy = level.ymid[:, None] - level.ymid[cand]
    keep = valid & (dx * dx + dy * dy < dist2)
    level.colleagues = _pack_rows(cand, keep)


def _gather_depths(levels):
    """Subtree depth of every node (numba_get_depths, flexmm/tree.py:362-369)."""
    L = len(levels)
    for ind in reversed(range(L)):
        lv = levels[ind]
        d = np.zeros(lv.n_node, dtype=np.int64)
        if ind < L - 1:
            inner = np.flatnonzero(~lv.leaf)
            if inner.size:
                ch = lv.children_ind[inner]
                dd = levels[ind + 1].depths
                d[inner] = np.max(np.stack([dd[ch + k] for k in range(4)]), axis=0) + 1
        lv.depths = d


def _colleague_depth_gap(lv, n_valid):
    """depth[i] - depth[c] for every colleague slot (huge where invalid)."""
    c = lv.colleagues[:n_valid]
    ok = (c >= 0) & (c < n_valid)
    dc = lv.depths[np.where(ok, c, 0)]
    gap = lv.depths[:n_valid, None] - dc
    return gap, ok


class Tree:
    """Adaptive quadtree over the sources (flexmm/tree.py:447-589)."""

    def __init__(self, x, y, ppl, bbox):
        self.x = np.array(x, dtype=np.float64)
        self.y = np.array(y, dtype=np.float64)
        self.points_per_leaf = ppl
        self.bbox = bbox
        self.xmin, self.xmax, self.ymin, self.ymax = (float(b) for b in bbox)
        self.N = self.x.shape[0]
        self.ordv = np.arange(self.N)
        width = self.xmax - self.xmin
        levels = [Level([self.xmin], [self.ymin], width, [0], [self.N], [-1])]
        # level-by-level refinement, flexmm/tree.py:191-220, 490-497
        if self.N > ppl:
            while True:
                cur = levels[-1]
                tosplit = cur.ns > ppl
                nx, ny, nb, nt, npar = _split(cur, tosplit, self.x, self.y, self.ordv, 0, False)
                new = Level(nx, ny, cur.half_width, nb, nt, npar)
                levels.append(new)
                if not np.any(new.ns > ppl):
                    break
        self.Levels = levels
        self.levels = len(levels)
        for ind, lv in enumerate(levels):
            _tag_colleagues(lv, None if ind == 0 else levels[ind - 1])
        _gather_depths(levels)
        self._level_restrict()
        self._split_xlist()
        self._post_process()
        self._build_interaction_lists()

    # -- flexmm/tree.py:529-541
    def _level_restrict(self):
        levels = self.Levels
        new_nodes = 1
        while new_nodes > 0:
            new_nodes = 0
            for ind in range(1, self.levels - 2):
                lv, desc = levels[ind], levels[ind + 1]
                gap, ok = _colleague_depth_gap(lv, lv.n_node)
                bads = lv.leaf & np.any(ok & ((gap > 1) | (gap < -1)), axis=1)
                out = _split(lv, bads, self.x, self.y, self.ordv, desc.n_node, False)
                desc.append(*out, fake=False)
                _tag_colleagues(desc, lv)
                _gather_depths(levels)
                new_nodes += int(bads.sum())

    # -- flexmm/tree.py:542-553, numba_get_Xlist flexmm/tree.py:385-397
    def _split_xlist(self):
        levels = self.Levels
        for ind, lv in enumerate(levels):
            lv.Xlist = np.zeros(lv.n_node, dtype=bool)
            if ind == 0 or ind == self.levels - 1:
                continue
            n_valid = lv.depths.shape[0]
            gap, ok = _colleague_depth_gap(lv, n_valid)
            lv.Xlist[:n_valid] = lv.leaf[:n_valid] & np.any(ok & (gap < 0), axis=1)
            if lv.Xlist.any():
                desc = levels[ind + 1]
                out = _split(lv, lv.Xlist, self.x, self.y, self.ordv, desc.n_node, True)
                desc.append(*out, fake=True)
                _tag_colleagues(desc, lv)

    # -- flexmm/tree.py:554-577
    def _post_process(self):
        for ind, lv in enumerate(self.Levels):
            lv.not_leaf = ~lv.leaf
            ns = lv.top_ind - lv.bot_ind
            lv.compute_upwards = (((lv.leaf & ~lv.Xlist) | lv.fake_leaf) & (ns > 0))
            lv.compute_downwards = ((lv.not_leaf | lv.Xlist) & ~lv.fake_leaf)
            lv.has_source = ns > 0
            if ind > 0:
                sib = lv.has_source.reshape(-1, 4).any(axis=1)
                lv.sib_has_source = sib
                lv.n_sib_has_source = int(sib.sum())
                lv.allocate_density = np.repeat(sib, 4)
                lv.n_allocate_density = int(lv.allocate_density.sum())
                lv.parent_density_ind = -np.ones(lv.n_node // 4, dtype=np.int64)
                lv.parent_density_ind[sib] = np.arange(lv.n_sib_has_source)
                lv.this_density_ind = -np.ones(lv.n_node, dtype=np.int64)
                lv.this_density_ind[lv.allocate_density] = np.arange(lv.n_allocate_density)

    # -- build_interaction_list, flexmm/tree.py:399-435, 582-589
    def _build_interaction_lists(self):
        self.interaction_lists = [None] * self.levels
        for ind in range(2, self.levels):
            lv, par = self.Levels[ind], self.Levels[ind - 1]
            n = lv.n_node
            dil = -np.ones((7, 7, n), dtype=np.int64)
            p = lv.parent_ind
            pc = par.colleagues[p]                                   # n x 9
            use = (pc >= 0) & (pc != p[:, None])
            pch = par.children_ind[np.where(use, pc, 0)]
            # the reference reads children_ind even for colleagues without
            # children (-1), giving node indices -1, 0, 1, 2 with numpy-style
            # wraparound; this only ever happens for fake leaves, whose local
            # expansions are never used, and is kept here for fidelity
            for j in range(9):
                for k in range(4):
                    ci = pch[:, j] + k
                    m = use[:, j]
                    ci_w = np.where(ci < 0, ci + n, ci)
                    xd = np.round((lv.xmid[ci_w] - lv.xmid) / lv.width).astype(np.int64)
                    yd = np.round((lv.ymid[ci_w] - lv.ymid) / lv.width).astype(np.int64)
                    di = lv.this_density_ind[ci_w]
                    ok = m & (di >= 0) & (np.abs(xd) <= 3) & (np.abs(yd) <= 3) \
                        & ~((np.abs(xd) <= 1) & (np.abs(yd) <= 1))
                    sel = np.flatnonzero(ok)
                    dil[xd[sel] + 3, yd[sel] + 3, sel] = di[sel]
            self.interaction_lists[ind] = dil

    def locate_points(self, x, y):
        """Root-to-leaf descent (numba_locate_points, flexmm/tree.py:712-727)."""
        x = np.ravel(x)
        y = np.ravel(y)
        inds = np.zeros(x.size, dtype=np.int64)
        locs = np.zeros(x.size, dtype=np.int64)
        active = np.flatnonzero(~self.Levels[0].leaf[locs])
        ind = 0
        while active.size:
            lv = self.Levels[ind]
            loc = locs[active]
            c = lv.children_ind[loc]
            c = c + 2 * (x[active] > lv.xmid[loc]) + (y[active] > lv.ymid[loc])
            ind += 1
            locs[active] = c
            inds[active] = ind
            active = active[~self.Levels[ind].leaf[c]]
        return inds, locs
