"""Canonical, numbering-independent description of a quadtree.

Two trees are equal when, level by level, they hold boxes at the same integer
positions with the same leaf / fake-leaf / X-list flags and point counts,
every source point sits in the same real leaf, colleague sets agree and the
far-field interaction lists name the same (target box, offset) pairs.  Node
order, the order of points inside a leaf and the order of colleague slots
are free to differ.

Works for both the oracle tree (``oracle.tree.Tree``) and the tree exported
by ``flexmm_b200`` (``FMM.tree``); both expose ``Levels[l]`` with ``xmin``,
``ymin``, ``width``, ``leaf``, ``fake_leaf``, ``Xlist``, ``bot_ind``,
``top_ind``, ``colleagues``, ``ordv`` and per-level interaction triples.
"""
import numpy as np


def _pos(lv, bbox):
    ix = np.rint((lv.xmin - bbox[0]) / lv.width).astype(np.int64)
    iy = np.rint((lv.ymin - bbox[2]) / lv.width).astype(np.int64)
    return ix, iy


def _sorted_rows(a):
    a = np.asarray(a, dtype=np.int64)
    if a.size == 0:
        return a.reshape(0, a.shape[1] if a.ndim == 2 else 0)
    return a[np.lexsort(a.T[::-1])]


def interaction_triples_from_dilists(tree, ind):
    """(target node, offset id 0..48, source node) from reference-style dilists."""
    lv = tree.Levels[ind]
    dil = tree.interaction_lists[ind]
    inv = -np.ones(lv.n_allocate_density, dtype=np.int64)
    alloc = np.flatnonzero(lv.this_density_ind >= 0)
    inv[lv.this_density_ind[alloc]] = alloc
    ii, jj, t = np.nonzero(dil >= 0)
    src = inv[dil[ii, jj, t]]
    return np.stack([t, ii * 7 + jj, src], axis=1)


def canonical(tree, triples_fn=interaction_triples_from_dilists, real_only=True,
              nonempty_sources=False):
    bbox = tree.bbox
    out = {"levels": len(tree.Levels)}
    leaf_of_point = np.full((tree.N, 3), -1, dtype=np.int64)
    for ind, lv in enumerate(tree.Levels):
        ix, iy = _pos(lv, bbox)
        xl = getattr(lv, "Xlist", np.zeros(lv.n_node, bool))
        ns = lv.top_ind - lv.bot_ind
        out[f"nodes{ind}"] = _sorted_rows(np.stack(
            [ix, iy, lv.leaf, lv.fake_leaf, xl, ns], axis=1))
        # every real leaf's points
        for n in np.flatnonzero(lv.leaf & ~lv.fake_leaf):
            pts = tree.ordv[lv.bot_ind[n]:lv.top_ind[n]]
            leaf_of_point[pts] = (ind, ix[n], iy[n])
        col = lv.colleagues
        i_idx, slot = np.nonzero(col >= 0)
        c = col[i_idx, slot]
        out[f"coll{ind}"] = _sorted_rows(np.stack([ix[i_idx], iy[i_idx], ix[c], iy[c]], axis=1))
        if ind >= 2:
            tr = triples_fn(tree, ind)
            if real_only and tr.size:
                tr = tr[~lv.fake_leaf[tr[:, 0]]]
            if nonempty_sources and tr.size:
                tr = tr[ns[tr[:, 2]] > 0]
            out[f"il{ind}"] = _sorted_rows(np.stack(
                [ix[tr[:, 0]], iy[tr[:, 0]], tr[:, 1], ix[tr[:, 2]], iy[tr[:, 2]]], axis=1)
                if tr.size else np.zeros((0, 5), np.int64))
    out["leaf_of_point"] = leaf_of_point
    return out


def gpu_triples(tree, ind):
    """Interaction triples of a flexmm_b200 TreeView."""
    return tree.interaction_triples(ind)


def compare(a, b):
    """Return a list of the canonical fields that differ (empty when equal)."""
    bad = []
    keys = sorted(set(a) | set(b), key=str)
    for k in keys:
        if k not in a or k not in b:
            bad.append(k)
            continue
        va, vb = np.asarray(a[k]), np.asarray(b[k])
        if va.shape != vb.shape or not np.array_equal(va, vb):
            bad.append(k)
    return bad
