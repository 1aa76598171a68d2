"""2D triangle meshes (UnstructuredMesh<Tri*>, the reference's TriMesh) on
the GPU, through the C-ABI, against the reference built from its sources:

  - triangle sub-boxes (17 per triangle: pick_binary_split<Simplex> and
    split_inplace<2,Simplex>, whose triangle index is the evaluators'
    layout) bit-exact against the reference's BVH at orders 1-3, which also
    pins the triangle faces of tet boundaries;
  - point location through LocateHack<2> (z ignored in the solve) against
    the reference's TriMesh locate; the persistent kernel bit-identical to
    the plain one;
  - field values at located points (drb_field_eval on a triangle field)
    against a closed-form Bernstein triangle evaluation.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _mesh(p):
    from devil_ray_b200 import meshgen
    return meshgen.tri_warped_mesh(20, p, 0.04, jitter=0.004, seed=5 + p)


def _gpu(m, cuda):
    from devil_ray_b200 import _lib as L
    from devil_ray_b200 import api
    return api.UnstructuredMesh(m.ctrl_idx, m.xyz, m.order, dim=2, device=cuda,
                                shape=L.SHAPE_SIMPLEX)


def _queries(n, seed):
    rng = np.random.default_rng(seed)
    xy = rng.uniform(-0.05, 1.05, size=(n, 2))
    return np.concatenate([xy, np.zeros((n, 1))], 1).astype(np.float32)


@pytest.mark.parametrize("p", [1, 2, 3])
def test_tri_subboxes_match_reference(cuda, ref, p):
    import torch
    from devil_ray_b200 import api
    from tests.bvh_util import subbox_aabbs
    m = _mesh(p)
    g = _gpu(m, cuda)
    aabbs, prim, refb, _ = api.elem_subboxes(g)
    torch.cuda.synchronize()
    rb = ref.RefTriMesh(p, m.ctrl_idx, m.xyz).bvh()
    ra = subbox_aabbs(rb["inner"], rb["aabb_ids"])
    assert np.array_equal(aabbs.cpu().numpy().view(np.int32), ra.view(np.int32))
    assert np.array_equal(refb.cpu().numpy().view(np.int32), rb["ref_boxes"].view(np.int32))


@pytest.mark.parametrize("p", [1, 2, 3])
def test_tri_locate_matches_reference(cuda, ref, p):
    import torch
    from devil_ray_b200 import _lib as L
    m = _mesh(p)
    g = _gpu(m, cuda)
    pts = _queries(60000, p)
    cell, rp = g.locate(pts, tol=1e-4, max_steps=20, guess_mode=L.GUESS_ZERO)
    torch.cuda.synchronize()
    cell, rp = cell.cpu().numpy(), rp.cpu().numpy()
    rc, rr = ref.RefTriMesh(p, m.ctrl_idx, m.xyz).locate(pts)
    same = cell == rc
    assert same.mean() > 0.999, f"{(~same).sum()} cell mismatches"
    both = same & (cell >= 0)
    assert np.abs(rp[both, :2] - rr[both, :2]).max() < 1e-3
    assert np.all(rp[cell >= 0, 2] == -1.0)
    assert 0.8 < (cell >= 0).mean() < 0.9


@pytest.mark.parametrize("p", [1, 2, 3])
@pytest.mark.parametrize("row_mode", [0, 1])
def test_tri_batched_identical_to_plain(cuda, p, row_mode):
    import torch
    from devil_ray_b200 import _lib as L
    from devil_ray_b200 import api
    m = _mesh(p)
    g = _gpu(m, cuda)
    pts = _queries(80000, 10 + p)
    c0, r0 = g.locate(pts, tol=1e-5, max_steps=20, guess_mode=L.GUESS_SUBREF_CENTER)
    cfg = L.DrbLocateConfig(128, 0, 64, 1, row_mode)
    c1, r1 = api.BatchedLocator(g, tol=1e-5, max_steps=20, guess_mode=L.GUESS_SUBREF_CENTER,
                                config=cfg).locate(pts)
    torch.cuda.synchronize()
    assert torch.equal(c0, c1)
    assert torch.equal(r0.view(torch.int32), r1.view(torch.int32))


@pytest.mark.parametrize("p", [1, 2, 3])
def test_tri_point_location_field_values(cuda, p):
    import torch
    from math import factorial
    from devil_ray_b200 import _lib as L
    from devil_ray_b200 import api
    from devil_ray_b200.render import PointLocation, QuadField
    m = _mesh(p)
    g = _gpu(m, cuda)
    f = QuadField(m.ctrl_idx, m.field, p, device=cuda, shape=L.SHAPE_SIMPLEX)
    pts = _queries(20000, 20 + p)
    q = PointLocation()
    q.add_var("f")
    q.empty_val(-3.0)
    vals = q.execute(g, {"f": f}, pts)["f"].cpu().numpy()
    cell, rp = api.BatchedLocator(g, 1e-4, 20).locate(pts)
    torch.cuda.synchronize()
    cell, rp = cell.cpu().numpy(), rp.cpu().numpy()
    assert np.all(vals[cell < 0] == np.float32(-3.0))
    nd = (p + 1) * (p + 2) // 2
    conn = m.ctrl_idx.reshape(-1, nd)
    sel = np.nonzero(cell >= 0)[0][:4000]
    u, v = rp[sel, 0].astype(np.float64), rp[sel, 1].astype(np.float64)
    t = 1 - u - v
    cv = m.field[conn[cell[sel]]].astype(np.float64)
    want = np.zeros(sel.size)
    for j in range(p + 1):
        for i in range(p + 1 - j):
            l = p - i - j
            B = factorial(p) / (factorial(i) * factorial(j) * factorial(l)) * u ** i * v ** j * t ** l
            want += B * cv[:, (2 * p + 3 - j) * j // 2 + i]
    assert np.abs(vals[sel] - want).max() < 1e-4
