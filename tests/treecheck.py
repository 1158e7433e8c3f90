"""Structural invariants of an exported LBVH, restating the reference's debug
kernels checkBVHIntegrity and checkPrimmap
(Mine/collision/lbvh/LBvhBuildKernels.cu:228-293) as vectorised checks.

tree: dict with inode (I x 6: lc, rc, par, mark, rangex, rangey), ibox (I x 6),
leaf (T x 4: orig id, par, mark, lca), lbox (T x 6), lca (T+1), primmap (T).
"""
import numpy as np


def check_tree(t, T):
    errs = []
    inode, leaf, lca, ibox, lbox = t["inode"], t["leaf"], t["lca"], t["ibox"], t["lbox"]
    I = T - 1
    if lca[T] != -1:
        errs.append("tail sentinel lca[T] != -1")
    # permutation validity (checkPrimmap)
    orig = leaf[:, 0]
    if not np.array_equal(np.sort(orig), np.arange(T)):
        errs.append("slot -> triangle map is not a permutation")
    if "primmap" in t and not np.array_equal(t["primmap"][orig], np.arange(T)):
        errs.append("primmap is not the inverse of the slot map")
    if T < 2:
        return errs
    lc, rc, par, mark, rx, ry = (inode[:, k] for k in range(6))
    # leaves as children
    lpar = leaf[:, 1]
    right = (leaf[:, 2] & 4) != 0
    s = np.arange(T)
    bad_r = right & ((rc[lpar] != s) | ((mark[lpar] & 2) == 0) | (ry[lpar] != s) |
                     ((lca[:T] & 1) == 0) | ((lca[:T] >> 1) != s))
    top = lca[:T] >> 1
    bad_l = (~right) & ((lc[lpar] != s) | ((mark[lpar] & 1) == 0) | (rx[lpar] != s) |
                        ((lca[:T] & 1) == 1))
    bad_l2 = (~right) & ((lca[:T] & 1) == 0)
    if bad_r.any():
        errs.append(f"{int(bad_r.sum())} right-child leaves inconsistent")
    if bad_l.any():
        errs.append(f"{int(bad_l.sum())} left-child leaves inconsistent")
    if bad_l2.any() and (rx[top[bad_l2]] != s[bad_l2]).any():
        errs.append("escape link of a left-child leaf is not its chain top")
    # internal nodes: DFS order, ranges, children
    d = np.arange(I)
    left_int = (mark & 1) == 0
    if (left_int & (lc != d + 1)).any():
        errs.append("internal left child is not the next DFS id")
    has_par = par >= 0
    if (par == -1).sum() != 1 or par[0] != -1:
        errs.append("root is not DFS id 0 or several roots")
    if (has_par & (par >= d)).any():
        errs.append("parent DFS id not smaller than child")
    # ranges: children partition the parent's range
    lo_l = np.where(mark & 1, lc, rx[np.clip(lc, 0, I - 1)])
    hi_l = np.where(mark & 1, lc, ry[np.clip(lc, 0, I - 1)])
    lo_r = np.where(mark & 2, rc, rx[np.clip(rc, 0, I - 1)])
    hi_r = np.where(mark & 2, rc, ry[np.clip(rc, 0, I - 1)])
    if ((lo_l != rx) | (hi_r != ry) | (hi_l + 1 != lo_r)).any():
        errs.append("child ranges do not partition the parent range")
    # right-child bit
    rbit = (mark & 4) != 0
    is_rc = np.zeros(I, bool)
    is_rc[rc[(mark & 2) == 0]] = True
    if (rbit[1:] != is_rc[1:]).any():
        errs.append("right-child mark bit inconsistent")
    # boxes: parent contains children
    cb_lo_l = np.where((mark & 1)[:, None], lbox[np.clip(lc, 0, T - 1), :3], ibox[np.clip(lc, 0, I - 1), :3])
    cb_lo_r = np.where((mark & 2)[:, None], lbox[np.clip(rc, 0, T - 1), :3], ibox[np.clip(rc, 0, I - 1), :3])
    cb_hi_l = np.where((mark & 1)[:, None], lbox[np.clip(lc, 0, T - 1), 3:], ibox[np.clip(lc, 0, I - 1), 3:])
    cb_hi_r = np.where((mark & 2)[:, None], lbox[np.clip(rc, 0, T - 1), 3:], ibox[np.clip(rc, 0, I - 1), 3:])
    if not (np.array_equal(ibox[:, :3], np.minimum(cb_lo_l, cb_lo_r)) and
            np.array_equal(ibox[:, 3:], np.maximum(cb_hi_l, cb_hi_r))):
        errs.append("internal box is not the exact union of its children")
    return errs


def pick_roots(tree, frac=0.25, lo=16, hi=512):
    """Disjoint subtrees (DFS ids) of lo..hi leaves covering about `frac` of
    the internal nodes: restructure marks for the tests."""
    inode = tree["inode"]
    size = inode[:, 5] - inode[:, 4] + 1
    covered = np.zeros(inode.shape[0] + 1, bool)
    chosen, total = [], 0
    for d in range(inode.shape[0]):
        if lo <= size[d] <= hi and not covered[d]:
            chosen.append(d)
            covered[d:d + size[d] - 1] = True
            total += size[d] - 1
            if total >= frac * inode.shape[0]:
                break
    return np.array(chosen, np.int32)
