"""CPU restatement of the adaptive octree / quadtree and its U / V / W / X
interaction lists, and the coverage property they must satisfy.  TEST
INFRASTRUCTURE.

The reference builds only uniform trees (cpu/morton_tree.cpp:286-493); the
adaptive tree has no reference counterpart, so this module restates its
rules directly from their definitions, by brute force over all cells, and
checks the property that makes an FMM exact up to truncation: for every
target leaf T and every source particle j, exactly one interaction accounts
for the pair (T, j):

* j lies in T or in a leaf of U(T)                    (near field, P2P)
* j lies in the subtree of a cell of W(T)             (M2P)
* j lies in a leaf of X(A), A = T or an ancestor      (P2L, then L2L down)
* j lies in the subtree of a cell of V(A), A as above (M2L, then L2L down)

Tree rules (the solver's, stated on integer cube coordinates): the adaptive
tree keeps the root of the uniform tree of `depth` levels and the children
of every kept cell that is split; a kept cell is split while it holds more
than max_leaf particles and lies above level depth - 1.  Two cubes touch
when they overlap or share a face, edge or corner.  For a cell B at level L:

* V(B): cells D at level L whose parent touches (or is) B's parent and that
  do not touch B (children of the parent's colleagues, not adjacent);
* U(B), B a leaf: leaves C != B of any level that touch B;
* W(B), B a leaf: cells D finer than B whose parent touches B and that do
  not touch B;
* X(B), L >= 2: leaves C at levels 1 .. L - 1 that touch B's parent and do
  not touch B (the transpose of W).

The uniform tree comes from the C restatement (oracle.Oracle.tree), pinned
to the reference's own tree by the golden fixtures.
"""
from __future__ import annotations

import numpy as np


def _coords(code: np.ndarray, dim: int = 3) -> np.ndarray:
    """Integer cube (square) coordinates of level-local Morton codes (bits
    x<<2 | y<<1 | z per level in 3D, x<<1 | y in 2D: the reference's
    interleave, cpu/morton_tree.cpp:48-99)."""
    code = np.asarray(code, dtype=np.uint64)
    out = np.zeros((len(code), dim), np.int64)
    for d in range(dim):
        v = code >> np.uint64(dim - 1 - d)
        r = np.zeros(len(code), np.int64)
        for b in range(64 // dim):
            r |= (((v >> np.uint64(dim * b)) & np.uint64(1)).astype(np.int64)) << b
        out[:, d] = r
    return out


def adaptive_from_uniform(tree: dict, max_leaf: int, dim: int = 3) -> dict:
    """The adaptive tree kept from a uniform tree (the oracle's export: per
    level code, child / particle ranges sb, se, parent) in the solver's
    numbering: kept cells level by level, in the uniform tree's order.
    Returns per cell: level, code, coords, parent (global, -1 root),
    pbeg, pend (tree positions), is_leaf; and the leaves in cell order."""
    levels = tree["levels"]
    D = len(levels)
    # particle ranges of every uniform cell, bottom up
    pb, pe = [None] * D, [None] * D
    pb[D - 1] = levels[D - 1]["sb"].copy()
    pe[D - 1] = levels[D - 1]["se"].copy()
    for L in range(D - 2, -1, -1):
        sb, se = levels[L]["sb"], levels[L]["se"]
        pb[L] = pb[L + 1][sb]
        pe[L] = pe[L + 1][se - 1]
    keep, split, gid = [], [], []
    cells = dict(level=[], code=[], parent=[], pbeg=[], pend=[], is_leaf=[])
    n_cells = 0
    for L in range(D):
        m = len(levels[L]["code"])
        if L == 0:
            k = np.ones(m, bool)
        else:
            par = levels[L]["parent"]
            k = keep[L - 1][par] & split[L - 1][par]
        cnt = pe[L] - pb[L]
        sp = k & (L < D - 1) & ((max_leaf == 0) | (cnt > max_leaf))
        g = np.full(m, -1, np.int64)
        g[k] = n_cells + np.arange(int(k.sum()))
        keep.append(k); split.append(sp); gid.append(g)
        n_cells += int(k.sum())
        idx = np.nonzero(k)[0]
        cells["level"].append(np.full(len(idx), L, np.int64))
        cells["code"].append(levels[L]["code"][idx].astype(np.uint64))
        cells["parent"].append(gid[L - 1][levels[L]["parent"][idx]] if L else np.full(len(idx), -1, np.int64))
        cells["pbeg"].append(pb[L][idx].astype(np.int64))
        cells["pend"].append(pe[L][idx].astype(np.int64))
        cells["is_leaf"].append(~sp[idx])
    out = {k_: np.concatenate(v) for k_, v in cells.items()}
    out["coords"] = _coords(out["code"], dim)
    out["leaves"] = np.nonzero(out["is_leaf"])[0]
    out["depth"] = D
    return out


def _touch_matrix(lc, cc, lb, cb):
    """touch[i, j]: cube i (level lc[i], coords cc[i]) and cube j (level
    lb[j] >= lc[i] assumed or not: both ways) overlap or share a boundary."""
    lc = np.asarray(lc)[:, None]; lb = np.asarray(lb)[None, :]
    fine = np.maximum(lc, lb)
    ok = np.ones((len(cc), len(cb)), bool)
    for d in range(cc.shape[1]):
        a0 = cc[:, d][:, None] << (fine - lc)
        a1 = (cc[:, d][:, None] + 1) << (fine - lc)
        b0 = cb[:, d][None, :] << (fine - lb)
        b1 = (cb[:, d][None, :] + 1) << (fine - lb)
        ok &= (a0 <= b1) & (b0 <= a1)
    return ok


def lists(cells: dict) -> dict:
    """U, W (rows = leaves, in the order of cells['leaves']), X and V (rows =
    cells) as lists of sorted global cell indices, by brute force."""
    lev, co, par, leaf = cells["level"], cells["coords"], cells["parent"], cells["is_leaf"]
    C = len(lev)
    T = _touch_matrix(lev, co, lev, co)
    parent_touch = np.zeros((C, C), bool)          # [b, d]: cell b touches parent(d)
    has_par = par >= 0
    parent_touch[:, has_par] = T[:, par[has_par]]
    U, W = [], []
    for b in cells["leaves"]:
        u = np.nonzero(leaf & T[b])[0]
        U.append(np.sort(u[u != b]))
        w = np.nonzero((lev > lev[b]) & parent_touch[b] & ~T[b])[0]
        W.append(np.sort(w))
    X, V = [], []
    for b in range(C):
        L = lev[b]
        if L < 2:
            X.append(np.zeros(0, np.int64)); V.append(np.zeros(0, np.int64))
            continue
        p = par[b]
        x = np.nonzero(leaf & (lev >= 1) & (lev <= L - 1) & T[:, p] & ~T[:, b])[0]
        X.append(np.sort(x))
        v = np.nonzero((lev == L) & parent_touch[p] & ~T[b])[0]
        V.append(np.sort(v))
    return dict(U=U, W=W, X=X, V=V)


def coverage(cells: dict, L: dict, n: int, send=None):
    """For every leaf T, how often each source particle (tree positions) is
    accounted for by the four kinds of interaction; returns (counts
    [leaves][n] as int8, source mask [n]).  send: per cell, the end of its
    sources (leaves hold sources first); None = every particle a source."""
    pb, pe, par = cells["pbeg"], cells["pend"], cells["parent"]
    src = np.ones(n, bool)
    if send is not None:
        src[:] = False
        for g in cells["leaves"]:
            src[pb[g]:send[g]] = True
    out = np.zeros((len(cells["leaves"]), n), np.int16)
    row_of_leaf = {int(g): i for i, g in enumerate(cells["leaves"])}
    for i, t in enumerate(cells["leaves"]):
        d = np.zeros(n + 1, np.int64)

        def add(cs):
            for c in cs:
                d[pb[c]] += 1
                d[pe[c]] -= 1
        add([t]); add(L["U"][i]); add(L["W"][i])
        a = t
        while a >= 0:
            add(L["X"][a]); add(L["V"][a])
            a = par[a]
        out[i] = np.cumsum(d)[:n]
    assert len(row_of_leaf) == len(cells["leaves"])
    return out, src


def assert_covered_once(cells: dict, L: dict, n: int, send=None):
    """Raise AssertionError naming the first (target leaf, source particle)
    pair that no interaction or more than one interaction accounts for."""
    cnt, src = coverage(cells, L, n, send)
    bad = (cnt != 1) & src[None, :]
    if bad.any():
        i, j = np.argwhere(bad)[0]
        raise AssertionError(f"target leaf {int(cells['leaves'][i])}: source at tree position {int(j)} "
                             f"covered {int(cnt[i, j])} times ({int(bad.sum())} pairs wrong)")
