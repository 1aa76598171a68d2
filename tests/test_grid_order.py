"""The property the grid candidate lists rest on, checked on the CPU against
the reference's own BVH (oracle/_ref, built from the reference sources).

DeviceMesh::locate (data_model/device_mesh.hpp:248-318) walks the LBVH
left child first, keeping the right child on a stack when the point lies in
both boxes, and tries a leaf's element when it reaches the leaf.  The grid
lists claim that the leaves it reaches for a point are exactly the leaves
whose own boxes hold the point, in sorted-leaf order, so that scanning the
point's grid cell (every leaf whose box overlaps the cell, in leaf order)
yields the same candidates in the same order.  Both halves are checked here
with the walk restated from that file: on random points, on points placed
exactly on leaf box faces and corners (where the <= / >= comparisons
decide), and outside the mesh; on the BVHs of hex (orders 2 and 3), tet,
quad and triangle meshes.  Points with a NaN coordinate are left out:
every box comparison with NaN is false, so the walk reaches every leaf
while the grid maps the point to its first cell; no solve converges for
such a point, so both give no cell."""
import numpy as np
import pytest

from tests.bvh_util import leaf_boxes, node_children

BARRIER = -2000000000


def _walk(inner4: np.ndarray, p) -> list:
    """Leaves in the order DeviceMesh::locate reaches them (no solve, so
    every reached leaf): inner4 is the node array as float4 records, node
    ids index float4s (4 per node), leaves are -(i + 1)."""
    out = []
    todo = [BARRIER]
    cur = 0
    while cur != BARRIER:
        if cur > -1:
            f, s, t = inner4[cur], inner4[cur + 1], inner4[cur + 2]
            in_left = not (p[0] < f[0] or p[1] < f[1] or p[2] < f[2]
                           or p[0] > f[3] or p[1] > s[0] or p[2] > s[1])
            in_right = not (p[0] < s[2] or p[1] < s[3] or p[2] < t[0]
                            or p[0] > t[1] or p[1] > t[2] or p[2] > t[3])
            if not in_left and not in_right:
                cur = todo.pop()
            else:
                kids = inner4[cur + 3].view(np.int32)
                cur = int(kids[0]) if in_left else int(kids[1])
                if in_left and in_right:
                    todo.append(int(kids[1]))
        else:
            out.append(-cur - 1)
            cur = todo.pop()
    return out


def _holds(lb: np.ndarray, p) -> np.ndarray:
    """Leaves whose box (xmin, xmax, ymin, ymax, zmin, zmax) holds p, with
    the node test's comparisons."""
    return ~((p[0] < lb[:, 0]) | (p[1] < lb[:, 2]) | (p[2] < lb[:, 4])
             | (p[0] > lb[:, 1]) | (p[1] > lb[:, 3]) | (p[2] > lb[:, 5]))


def _axis(x, o, inv, g):
    """Grid cell along one axis: floor((x - o) * inv) clamped to [0, g - 1]."""
    v = np.float32(np.float32(x) - np.float32(o)) * np.float32(inv)
    return int(np.floor(min(max(np.float32(v), np.float32(0)), np.float32(g - 1))))


def _grid(lb: np.ndarray, o, inv, g):
    """Cell -> leaves whose box overlaps it, in leaf order."""
    cells = {}
    for k in range(lb.shape[0]):
        r = [range(_axis(lb[k, 2 * d], o[d], inv[d], g[d]),
                   _axis(lb[k, 2 * d + 1], o[d], inv[d], g[d]) + 1) for d in range(3)]
        for cz in r[2]:
            for cy in r[1]:
                for cx in r[0]:
                    cells.setdefault((cx, cy, cz), []).append(k)
    return cells


@pytest.mark.parametrize("name", ["trilinear_6", "warped_p3_4", "tet_p2", "quad_p2", "tri_p2"])
def test_walk_order_is_leaf_order_and_grid_scan_matches(ref, name):
    from devil_ray_b200 import meshgen
    flat = name in ("quad_p2", "tri_p2")
    if name == "trilinear_6":
        m = meshgen.trilinear_distorted_mesh(6, 2, 0.15, seed=11)
        b = ref.RefHexMesh(m.order, m.ctrl_idx, m.xyz).bvh()
    elif name == "warped_p3_4":
        m = meshgen.warped_mesh(4, 3, 0.08, jitter=0.01, seed=5)
        b = ref.RefHexMesh(m.order, m.ctrl_idx, m.xyz).bvh()
    elif name == "tet_p2":
        m = meshgen.tet_warped_mesh(3, 2, 0.05, jitter=0.01, seed=5)
        b = ref.RefTetMesh(m.order, m.ctrl_idx, m.xyz).bvh()
    elif name == "quad_p2":
        m = meshgen.quad_warped_mesh(8, 2, 0.04, jitter=0.004, seed=9)
        b = ref.RefQuadMesh(m.order, m.ctrl_idx, m.xyz).bvh()
    else:
        m = meshgen.tri_warped_mesh(6, 2, 0.04, jitter=0.004, seed=9)
        b = ref.RefTriMesh(m.order, m.ctrl_idx, m.xyz).bvh()
    inner = b["inner"]
    n_leaf = b["leaf_nodes"].shape[0]
    inner4 = inner.reshape(-1, 4)
    lb = leaf_boxes(inner, n_leaf)
    assert not np.isnan(lb).any()
    l, r = node_children(inner)
    assert ((l < 0).sum() + (r < 0).sum()) == n_leaf

    rng = np.random.default_rng(7)
    pts = [rng.uniform(-0.05, 1.05, 3).astype(np.float32) for _ in range(1500)]
    if flat:
        # 2D meshes lie in z = 0: most queries on the plane, some off it
        for q in pts[:1300]:
            q[2] = 0.0
    # on leaf box faces and corners: coordinates taken from the boxes
    for k in rng.choice(n_leaf, 300, replace=False):
        q = rng.uniform(lb[k, 0::2], lb[k, 1::2]).astype(np.float32)
        d = rng.integers(0, 3)
        q[d] = lb[k, 2 * d + rng.integers(0, 2)]
        pts.append(q)
        pts.append(lb[k, [0, 2, 4]].copy())
        pts.append(lb[k, [1, 3, 5]].copy())
    pts.append(np.array([5.0, 5.0, 5.0], np.float32))
    pts.append(np.array([-np.inf, 0.5, 0.5], np.float32))

    # a grid over the bounds with cells of about one mean leaf extent
    bounds = b["bounds"]
    o = bounds[0::2].astype(np.float32)
    ext = (lb[:, 1::2] - lb[:, 0::2]).mean(axis=0)
    span = [float(bounds[2 * d + 1] - bounds[2 * d]) for d in range(3)]
    g = [max(1, int(np.ceil(span[d] / ext[d]))) if ext[d] > 0 and span[d] > 0 else 1
         for d in range(3)]
    inv = [np.float32(g[d] / span[d]) if span[d] > 0 else np.float32(0) for d in range(3)]
    cells = _grid(lb, o, inv, g)

    reached = 0
    for p in pts:
        walk = _walk(inner4, p)
        held = np.flatnonzero(_holds(lb, p)).tolist()
        assert walk == held, (p, walk, held)
        c = tuple(_axis(p[d], o[d], inv[d], g[d]) for d in range(3))
        scan = [k for k in cells.get(c, []) if _holds(lb[k:k + 1], p)[0]]
        assert scan == walk, (p, scan, walk)
        reached += len(walk)
    assert reached > len(pts)  # most points meet at least one leaf, many several
