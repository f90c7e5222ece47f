"""Test helpers: read the device tree through the C ABI, compare trees."""
import ctypes

import numpy as np

P = ctypes.c_void_p


def ptr(a):
    return a.ctypes.data_as(P) if a is not None else None


def gpu_tree(ctx, dim, pts, q, depth, targets=None):
    """Build the uniform tree on the GPU (sources pts/q, optional targets) and
    read every level back, in the same dict layout as the oracle's export."""
    L = ctx.lib
    pts = np.ascontiguousarray(pts, dtype=np.float64)
    q = np.ascontiguousarray(q, dtype=np.float64)
    nt = 0 if targets is None else len(targets)
    tg = None if targets is None else np.ascontiguousarray(targets, dtype=np.float64)
    sizes = np.zeros(32, np.uint64)
    tnum = ctypes.c_size_t()
    ctx.check(L.lfmm_tree_build(ctx.handle, dim, len(pts), ptr(pts), ptr(q), nt, ptr(tg), depth, ptr(sizes),
                                ctypes.byref(tnum)), "tree_build")
    levels = []
    for lvl in range(depth):
        m = int(sizes[lvl])
        code = np.zeros(m, np.uint64)
        sb, se, tb, te, par = (np.zeros(m, np.int64) for _ in range(5))
        cen = np.zeros((m, dim))
        ctx.check(L.lfmm_tree_level(ctx.handle, lvl, ptr(code), ptr(sb), ptr(se), ptr(tb), ptr(te), ptr(par),
                                    ptr(cen)), "tree_level")
        nc = np.zeros(m, np.int64); nf = np.zeros(m, np.int64)
        ctx.check(L.lfmm_tree_list_sizes(ctx.handle, lvl, ptr(nc), ptr(nf)), "list_sizes")
        close = np.zeros(int(nc.sum()), np.int64)
        far = np.zeros(int(nf.sum()), np.int64)
        ctx.check(L.lfmm_tree_lists(ctx.handle, lvl, ptr(close), ptr(far)), "lists")
        levels.append(dict(code=code, sb=sb, se=se, tb=tb, te=te, parent=par, center=cen,
                           close_off=np.concatenate([[0], np.cumsum(nc)]), close=close,
                           far_off=np.concatenate([[0], np.cumsum(nf)]), far=far))
    pos = np.zeros(len(pts) + nt, np.int64)
    ctx.check(L.lfmm_tree_positions(ctx.handle, ptr(pos)), "positions")
    return dict(levels=levels, positions=pos, targets_num=tnum.value)


def leaf_members(tree, n):
    """Per leaf: (sorted input indices of sources, of targets)."""
    inv = np.empty(n, np.int64)
    inv[tree["positions"]] = np.arange(n)
    lv = tree["levels"][-1]
    out = []
    for c in range(len(lv["code"])):
        s = np.sort(inv[lv["sb"][c]:lv["se"][c]])
        t = np.sort(inv[lv["tb"][c]:lv["te"][c]]) if tree["targets_num"] else np.zeros(0, np.int64)
        out.append((s, t))
    return out


def assert_trees_equal(a, b, n, exact_positions=True, check_far=True):
    """Integer fields bit-exact, lists equal in order, centres exact."""
    assert a["targets_num"] == b["targets_num"]
    D = len(a["levels"])
    assert D == len(b["levels"])
    for L in range(D):
        A, B = a["levels"][L], b["levels"][L]
        np.testing.assert_array_equal(A["code"], B["code"], err_msg=f"codes, level {L}")
        if L < D - 1 or a["targets_num"] == 0:
            np.testing.assert_array_equal(A["sb"], B["sb"], err_msg=f"ranges, level {L}")
            np.testing.assert_array_equal(A["se"], B["se"], err_msg=f"ranges, level {L}")
        if L > 0:
            np.testing.assert_array_equal(A["parent"], B["parent"], err_msg=f"parents, level {L}")
        np.testing.assert_array_equal(A["close_off"], B["close_off"], err_msg=f"close counts, level {L}")
        np.testing.assert_array_equal(A["close"], B["close"], err_msg=f"close lists, level {L}")
        if check_far:
            np.testing.assert_array_equal(A["far_off"], B["far_off"], err_msg=f"far counts, level {L}")
            np.testing.assert_array_equal(A["far"], B["far"], err_msg=f"far lists, level {L}")
    if exact_positions:
        np.testing.assert_array_equal(a["positions"], b["positions"])
    else:
        ma, mb = leaf_members(a, n), leaf_members(b, n)
        assert len(ma) == len(mb)
        for (sa, ta), (sb_, tb_) in zip(ma, mb):
            np.testing.assert_array_equal(sa, sb_)
            np.testing.assert_array_equal(ta, tb_)


def gpu_adaptive_tree(ctx, pts, q, depth, max_leaf, targets=None, dim=3):
    """Build the adaptive tree (octree, or quadtree with dim = 2) on the GPU
    and read its cells and U / W / X / V lists back (CSR, global cell
    indices), in the layout of oracle/adaptive.py."""
    L = ctx.lib
    pts = np.ascontiguousarray(pts, dtype=np.float64)
    q = np.ascontiguousarray(q, dtype=np.float64)
    nt = 0 if targets is None else len(targets)
    tg = None if targets is None else np.ascontiguousarray(targets, dtype=np.float64)
    nc, nl = ctypes.c_size_t(), ctypes.c_size_t()
    sizes = np.zeros(4, np.uint64)
    build = L.lfmm_tree_build_adaptive if dim == 3 else L.lfmm2d_tree_build_adaptive
    ctx.check(build(ctx.handle, len(pts), ptr(pts), ptr(q), nt, ptr(tg), depth, max_leaf,
                    ctypes.byref(nc), ctypes.byref(nl), ptr(sizes)), "tree_build_adaptive")
    C, NL = nc.value, nl.value
    level = np.zeros(C, np.int32)
    code = np.zeros(C, np.uint64)
    parent, pbeg, pend, send = (np.zeros(C, np.int64) for _ in range(4))
    leaf = np.zeros(C, np.uint8)
    leaves = np.zeros(NL, np.int64)
    pos = np.zeros(len(pts) + nt, np.int64)
    ctx.check(L.lfmm_tree_adaptive_cells(ctx.handle, ptr(level), ptr(code), ptr(parent), ptr(pbeg), ptr(pend),
                                         ptr(send), ptr(leaf), ptr(leaves), ptr(pos)), "adaptive_cells")
    lists = {}
    for kind, name in enumerate("UWXV"):
        rows = NL if kind < 2 else C
        off = np.zeros(rows + 1, np.int64)
        idx = np.zeros(int(sizes[kind]), np.int64)
        ctx.check(L.lfmm_tree_adaptive_lists(ctx.handle, kind, ptr(off), ptr(idx)), "adaptive_lists")
        lists[name] = [np.sort(idx[off[r]:off[r + 1]]) for r in range(rows)]
    cells = dict(level=level.astype(np.int64), code=code, parent=parent, pbeg=pbeg, pend=pend,
                 is_leaf=leaf.astype(bool), leaves=leaves)
    return cells, lists, send, pos
