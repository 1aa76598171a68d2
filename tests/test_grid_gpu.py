"""Uniform-grid candidate lists (drb_bvh_grid_size / drb_bvh_grid_build).

* the lists against a NumPy restatement from the leaf boxes read out of the
  binary nodes: every cell holds exactly the leaves whose boxes overlap it,
  in leaf order, and the box table holds each leaf's box and element;
* the batched locate over the grid against the same locate over the 4-wide
  tree: cells, reference points, Newton iterations and candidates equal
  bit for bit (the grid yields the traversal's candidates in its order), on
  hex and tet meshes, at several cell sizes and first guesses.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _mesh(name):
    from devil_ray_b200 import _lib as L
    from devil_ray_b200 import meshgen
    if name == "trilinear_12":
        return meshgen.trilinear_distorted_mesh(12, 2, 0.15, seed=11), L.SHAPE_TENSOR
    if name == "p3_10":
        return meshgen.warped_mesh(10, 3, 0.08, jitter=0.01, seed=5), L.SHAPE_TENSOR
    if name == "p1_9":
        return meshgen.warped_mesh(9, 1, 0.05), L.SHAPE_TENSOR
    if name == "tet_p2":
        return meshgen.tet_warped_mesh(6, 2, 0.05, jitter=0.01, seed=5), L.SHAPE_SIMPLEX
    raise ValueError(name)


def _gpu(cuda, name):
    from devil_ray_b200 import api
    m, shape = _mesh(name)
    return m, api.UnstructuredMesh(m.ctrl_idx, m.xyz, m.order, device=cuda, shape=shape)


def _axis(x, o, inv, g):
    v = (np.float32(x) - np.float32(o)).astype(np.float32) * np.float32(inv)
    v = np.minimum(np.maximum(v.astype(np.float32), np.float32(0)), np.float32(g - 1))
    return np.floor(v).astype(np.int64)


@pytest.mark.parametrize("name,scale", [("trilinear_12", 1.0), ("p1_9", 0.5), ("tet_p2", 2.0)])
def test_grid_lists_match_restatement(cuda, name, scale):
    import torch
    from tests.bvh_util import leaf_boxes
    _, g = _gpu(cuda, name)
    b = g.get_bvh().build_grid(scale)
    torch.cuda.synchronize()
    dims, origin, inv = b.grid_geom
    lb = leaf_boxes(b.inner_nodes.cpu().numpy(), b.n_leaf)  # xmin,xmax,ymin,ymax,zmin,zmax
    lo, hi = lb[:, [0, 2, 4]], lb[:, [1, 3, 5]]
    c0 = np.stack([_axis(lo[:, d], origin[d], inv[d], dims[d]) for d in range(3)], 1)
    c1 = np.stack([_axis(hi[:, d], origin[d], inv[d], dims[d]) for d in range(3)], 1)
    keys, vals = [], []
    for k in range(b.n_leaf):
        zz, yy, xx = np.meshgrid(np.arange(c0[k, 2], c1[k, 2] + 1), np.arange(c0[k, 1], c1[k, 1] + 1),
                                 np.arange(c0[k, 0], c1[k, 0] + 1), indexing="ij")
        cells = ((zz * dims[1] + yy) * dims[0] + xx).ravel()
        keys.append(cells)
        vals.append(np.full(cells.size, k))
    keys, vals = np.concatenate(keys), np.concatenate(vals)
    order = np.lexsort((vals, keys))
    keys, vals = keys[order], vals[order]
    n_cells = dims[0] * dims[1] * dims[2]
    start = np.searchsorted(keys, np.arange(n_cells + 1), side="left")
    assert np.array_equal(b.grid_start.cpu().numpy(), start.astype(np.int32))
    ent = b.grid_entries.cpu().numpy()
    assert np.array_equal(ent, vals.astype(np.int32))
    box = b.grid_boxes.cpu().numpy()
    assert np.array_equal(box[:, [0, 1, 2]], lo) and np.array_equal(box[:, [4, 5, 6]], hi)
    assert np.array_equal(box[:, 3].view(np.int32), b.leaf_nodes.cpu().numpy())
    assert np.all(box[:, 7] == 0)
    print(f"{name}: {dims} cells, {keys.size} entries, {keys.size / n_cells:.2f} per cell")


@pytest.mark.parametrize("name", ["trilinear_12", "p3_10", "p1_9", "tet_p2"])
@pytest.mark.parametrize("scale", [0.5, 1.0, 3.0])
def test_grid_locate_equals_tree(cuda, name, scale):
    import torch
    from devil_ray_b200 import _lib as L
    from devil_ray_b200 import api, meshgen
    m, g = _gpu(cuda, name)
    q = meshgen.uniform_queries(80000, 91)
    bvh = g.get_bvh()
    tree = bvh.without_grid()
    grid = bvh.without_grid().build_grid(scale)
    modes = [L.GUESS_ELEM_CENTER, L.GUESS_SUBBOX_LINEAR] if scale == 1.0 else [L.GUESS_SUBREF_CENTER]
    for mode in modes:
        out = []
        for b in (tree, grid):
            if mode == L.GUESS_SUBBOX_LINEAR and b.leaf_maps is None:
                b.build_leaf_maps(g)
            loc = api.BatchedLocator(g, tol=1e-5, max_steps=20, guess_mode=mode, bvh=b)
            out.append(loc.locate(q, stats=True))
        torch.cuda.synchronize()
        (c0, r0, i0, a0, _), (c1, r1, i1, a1, n1) = out
        assert torch.equal(c0, c1)
        assert torch.equal(r0.view(torch.int32), r1.view(torch.int32))
        assert torch.equal(i0, i1) and torch.equal(a0, a1)
        assert (c1 >= 0).float().mean() > 0.5
        print(f"{name} scale {scale} mode {mode}: entries tested per query "
              f"{float(n1.float().mean()):.2f}")


def test_grid_rejects_bad_calls(cuda):
    import ctypes as C
    from devil_ray_b200 import _lib as L
    m = C.c_longlong()
    _, g = _gpu(cuda, "p1_9")
    bd = g.get_bvh().desc()
    assert L.lib().drb_bvh_grid_size(C.byref(bd), 0.0, C.byref(m), None) == L.DRB_ERR_INVALID_ARG
    # no lists set: build refuses
    assert L.lib().drb_bvh_grid_build(C.byref(bd), None) == L.DRB_ERR_INVALID_ARG


def test_grid_locate_edge_cases(cuda):
    """Empty batches, points far outside, on the bounds, at infinity and with
    a NaN coordinate: the grid path returns what the tree walk returns."""
    import torch
    from devil_ray_b200 import _lib as L
    from devil_ray_b200 import api
    _, g = _gpu(cuda, "trilinear_12")
    bvh = g.get_bvh()
    grid = bvh.without_grid().build_grid(0.75)
    tree = api.BatchedLocator(g, tol=1e-5, max_steps=20, bvh=bvh.without_grid())
    fast = api.BatchedLocator(g, tol=1e-5, max_steps=20, bvh=grid)
    c, r = fast.locate(np.zeros((0, 3), np.float32))
    assert c.numel() == 0
    pts = np.array([[5, 5, 5], [-1, 0.5, 0.5], [np.nan, 0.5, 0.5], [0.5, np.inf, 0.5],
                    [-np.inf, 0.2, 0.2], [0, 0, 0], [1, 1, 1], [0.5, 0.5, 0.5],
                    [1e30, -1e30, 0.5]], np.float32)
    c0, r0 = tree.locate(pts)
    c1, r1 = fast.locate(pts)
    torch.cuda.synchronize()
    assert torch.equal(c0, c1)
    assert torch.equal(r0.view(torch.int32), r1.view(torch.int32))
    c1 = c1.cpu().numpy()
    assert (c1[:5] == -1).all() and c1[8] == -1 and c1[7] >= 0


@pytest.mark.parametrize("kind", ["quad", "tri"])
def test_grid_locate_equals_tree_2d(cuda, kind):
    """2D quad and triangle meshes (their boxes are flat in z, so the grid
    has one cell across z): grid and tree give the same answers bit for
    bit, with queries on and off the mesh plane."""
    import torch
    from devil_ray_b200 import _lib as L
    from devil_ray_b200 import api, meshgen
    if kind == "quad":
        m = meshgen.quad_warped_mesh(24, 2, 0.04, jitter=0.004, seed=9)
        g = api.UnstructuredMesh(m.ctrl_idx, m.xyz, 2, dim=2, device=cuda)
    else:
        m = meshgen.tri_warped_mesh(16, 2, 0.04, jitter=0.004, seed=9)
        g = api.UnstructuredMesh(m.ctrl_idx, m.xyz, 2, dim=2, device=cuda, shape=L.SHAPE_SIMPLEX)
    rng = np.random.default_rng(3)
    xy = rng.uniform(-0.05, 1.05, size=(50000, 2))
    z = np.where(rng.random(50000) < 0.9, 0.0, 0.01)
    q = np.concatenate([xy, z[:, None]], 1).astype(np.float32)
    bvh = g.get_bvh()
    tree = api.BatchedLocator(g, tol=1e-5, max_steps=20, bvh=bvh.without_grid())
    grid = api.BatchedLocator(g, tol=1e-5, max_steps=20, bvh=bvh.without_grid().build_grid(1.0))
    c0, r0, i0, a0, _ = tree.locate(q, stats=True)
    c1, r1, i1, a1, _ = grid.locate(q, stats=True)
    torch.cuda.synchronize()
    assert grid.bvh.grid_geom[0][2] == 1
    assert torch.equal(c0, c1) and torch.equal(r0.view(torch.int32), r1.view(torch.int32))
    assert torch.equal(i0, i1) and torch.equal(a0, a1)
    assert (c1 >= 0).float().mean() > 0.5
