"""Helpers to read BVHs in the reference layout (bvh.hpp:16-37) for parity
checks: node children, leaf boxes by sub-box id, tie runs of Morton codes."""
from __future__ import annotations

import numpy as np


def node_children(inner: np.ndarray):
    """(left, right) child ids of every inner node, as the int bits of
    floats 12 and 13: inner child = 4*node, leaf = -(i+1)."""
    kids = np.ascontiguousarray(inner[:, 12:14]).view(np.int32)
    return kids[:, 0].copy(), kids[:, 1].copy()


def node_boxes(inner: np.ndarray):
    """Left and right child boxes of every node as (xmin,xmax,ymin,ymax,zmin,zmax)."""
    lb = inner[:, [0, 3, 1, 4, 2, 5]]
    rb = inner[:, [6, 9, 7, 10, 8, 11]]
    return lb, rb


def leaf_boxes(inner: np.ndarray, n_leaf: int) -> np.ndarray:
    """AABB of every sorted leaf, recovered from its parent's node record."""
    l, r = node_children(inner)
    lb, rb = node_boxes(inner)
    out = np.full((n_leaf, 6), np.nan, np.float32)
    m = l < 0
    out[-l[m] - 1] = lb[m]
    m = r < 0
    out[-r[m] - 1] = rb[m]
    return out


def subbox_aabbs(inner: np.ndarray, aabb_ids: np.ndarray) -> np.ndarray:
    """Per-sub-box AABBs in the original (element-major) order."""
    n_leaf = aabb_ids.shape[0]
    lbx = leaf_boxes(inner, n_leaf)
    out = np.empty_like(lbx)
    out[aabb_ids] = lbx
    return out


def tie_runs(sorted_codes: np.ndarray):
    """(start, end) of every run of >=2 equal codes in a sorted array."""
    c = np.asarray(sorted_codes)
    if c.size == 0:
        return []
    change = np.flatnonzero(np.diff(c) != 0) + 1
    starts = np.concatenate([[0], change])
    ends = np.concatenate([change, [c.size]])
    return [(int(s), int(e)) for s, e in zip(starts, ends) if e - s > 1]


def node_leaf_ranges(inner: np.ndarray):
    """[first, last] sorted-leaf range covered by each inner node."""
    l, r = node_children(inner)
    n_inner = inner.shape[0]
    lo = np.full(n_inner, -1, np.int64)
    hi = np.full(n_inner, -1, np.int64)
    # iterative post-order from the root
    order = []
    stack = [0]
    while stack:
        n = stack.pop()
        order.append(n)
        for c in (l[n], r[n]):
            if c >= 0:
                stack.append(c // 4)
    for n in reversed(order):
        ranges = []
        for c in (l[n], r[n]):
            if c < 0:
                ranges.append((-c - 1, -c - 1))
            else:
                ranges.append((lo[c // 4], hi[c // 4]))
        lo[n] = min(a for a, _ in ranges)
        hi[n] = max(b for _, b in ranges)
    return lo, hi


def widen(inner: np.ndarray):
    """Reference collapse of a binary BVH into the 4-wide tree the CUDA path
    builds: every inner node at even depth keeps its grandchildren (or its
    children where those are leaves) left to right.  Returns (boxes
    [n_wide, 4, 6] as xmin,xmax,ymin,ymax,zmin,zmax, codes [n_wide, 4]) with
    wide nodes numbered in binary-node order, empty slots code INT_MIN."""
    l, r = node_children(inner)
    lb, rb = node_boxes(inner)
    n = inner.shape[0]
    depth = np.full(n, -1, np.int64)
    depth[0] = 0
    stack = [0]
    while stack:
        i = stack.pop()
        for c in (l[i], r[i]):
            if c >= 0:
                depth[c // 4] = depth[i] + 1
                stack.append(c // 4)
    wide = np.where(depth % 2 == 0)[0]
    wid = np.full(n, -1, np.int64)
    wid[wide] = np.arange(wide.size)
    boxes = np.zeros((wide.size, 4, 6), np.float32)
    boxes[:, :, [0, 2, 4]] = np.inf
    boxes[:, :, [1, 3, 5]] = -np.inf
    codes = np.full((wide.size, 4), np.iinfo(np.int32).min, np.int64)
    for w, i in enumerate(wide):
        k = 0
        for c, b in ((l[i], lb[i]), (r[i], rb[i])):
            if c < 0:
                boxes[w, k], codes[w, k] = b, c
                k += 1
            else:
                j = c // 4
                for g, gb in ((l[j], lb[j]), (r[j], rb[j])):
                    boxes[w, k] = gb
                    codes[w, k] = g if g < 0 else wid[g // 4]
                    k += 1
    return boxes, codes.astype(np.int32)


def leaf_maps_fp64(shape: str, p: int, ctrl_idx, xyz, bvh, leaves):
    """FP64 restatement of drb_bvh_leaf_maps for the given sorted leaves:
    (c, X(c), J(c)^-1 row-major) with c the sub-box centre (hex) or the mean
    of the sub-simplex's four vertices (tet), in the float32 arithmetic of
    the kernel."""
    from oracle import restate
    nd = (p + 1) ** 3 if shape == "hex" else (p + 1) * (p + 2) * (p + 3) // 6
    ci = np.asarray(ctrl_idx).reshape(-1, nd)
    els = bvh.leaf_nodes.cpu().numpy()[leaves]
    ids = bvh.aabb_ids.cpu().numpy()[leaves]
    rb = bvh.ref_boxes.cpu().numpy()
    out = np.zeros((len(leaves), 15))
    for k, (e, a) in enumerate(zip(els, ids)):
        if shape == "hex":
            b = rb.reshape(-1, 6)[a]
            c = ((b[:3] + b[3:]) * np.float32(0.5)).astype(np.float32)
            X, J = restate.hex_eval_d(p, xyz[ci[e]], c)
        else:
            b = rb.reshape(-1, 12)[a].reshape(4, 3)
            c = ((b[0] + b[1] + b[2] + b[3]) * np.float32(0.25)).astype(np.float32)
            X, J = restate.tet_eval_d(p, xyz[ci[e]], c)
        out[k, :3] = c
        out[k, 3:6] = X[0]
        out[k, 6:] = np.linalg.inv(J[0].T).ravel()
    return out
