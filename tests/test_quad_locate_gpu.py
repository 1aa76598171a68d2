"""Point location on 2D (quad) meshes: UnstructuredMesh<Quad*>::locate
through LocateHack<2> (data_model/device_mesh.hpp:166-238), where z is
ignored (the 3x3 Jacobian's third column is e_z), against the reference
built from its sources (oracle/_ref), through the C-ABI (drb_locate,
drb_locate_batched on a dim-2 mesh) and drb_field_eval on a quad field.

Tolerances: cells identical on >= 99.9 % of queries, reference coordinates
within 1e-3 of the reference (the third stays -1 as in the reference's
Location), field values within 1e-4 of a closed-form tensor Bernstein
evaluation.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _mesh(p):
    from devil_ray_b200 import meshgen
    return meshgen.quad_warped_mesh(24, p, 0.04, jitter=0.004, seed=7 + p)


def _queries(n, seed, z=0.0):
    rng = np.random.default_rng(seed)
    xy = rng.uniform(-0.05, 1.05, size=(n, 2))
    return np.concatenate([xy, np.full((n, 1), z)], 1).astype(np.float32)


def _bern(p, t):
    from math import comb
    return np.stack([comb(p, i) * t ** i * (1 - t) ** (p - i) for i in range(p + 1)], -1)


@pytest.mark.parametrize("p", [1, 2, 3])
def test_quad_locate_matches_reference(cuda, ref, p):
    import torch
    from devil_ray_b200 import _lib as L
    from devil_ray_b200 import api
    m = _mesh(p)
    g = api.UnstructuredMesh(m.ctrl_idx, m.xyz, p, dim=2, device=cuda)
    pts = _queries(60000, p)
    cell, rp = g.locate(pts, tol=1e-4, max_steps=20, guess_mode=L.GUESS_ZERO)
    torch.cuda.synchronize()
    cell, rp = cell.cpu().numpy(), rp.cpu().numpy()
    rc, rr = ref.RefQuadMesh(p, m.ctrl_idx, m.xyz).locate(pts)
    same = cell == rc
    assert same.mean() > 0.999, f"{(~same).sum()} cell mismatches"
    both = same & (cell >= 0)
    assert np.abs(rp[both, :2] - rr[both, :2]).max() < 1e-3
    assert np.all(rp[cell >= 0, 2] == -1.0)
    assert 0.8 < (cell >= 0).mean() < 0.9


@pytest.mark.parametrize("p", [1, 2, 3])
@pytest.mark.parametrize("row_mode", [0, 1])
def test_quad_batched_identical_to_plain(cuda, p, row_mode):
    import torch
    from devil_ray_b200 import _lib as L
    from devil_ray_b200 import api
    m = _mesh(p)
    g = api.UnstructuredMesh(m.ctrl_idx, m.xyz, p, dim=2, device=cuda)
    pts = _queries(80000, 10 + p)
    c0, r0 = g.locate(pts, tol=1e-5, max_steps=20, guess_mode=L.GUESS_ELEM_CENTER)
    cfg = L.DrbLocateConfig()
    cfg.block, cfg.blocks_per_sm, cfg.chunk, cfg.sort_queries, cfg.reg_elements = 128, 0, 64, 1, row_mode
    c1, r1 = api.BatchedLocator(g, tol=1e-5, max_steps=20, config=cfg).locate(pts)
    torch.cuda.synchronize()
    assert torch.equal(c0, c1)
    assert torch.equal(r0.view(torch.int32), r1.view(torch.int32))


def test_quad_locate_off_plane_queries(cuda, ref):
    """The Newton solve ignores z, but the BVH's point-in-box test does not:
    the boxes of a flat mesh have zero z extent, so a query off the mesh's
    plane is not located, by the reference either."""
    import torch
    from devil_ray_b200 import api
    m = _mesh(2)
    g = api.UnstructuredMesh(m.ctrl_idx, m.xyz, 2, dim=2, device=cuda)
    q = _queries(20000, 3, 0.37)
    c1, _ = api.BatchedLocator(g).locate(q)
    torch.cuda.synchronize()
    rc, _ = ref.RefQuadMesh(2, m.ctrl_idx, m.xyz).locate(q)
    assert np.all(rc == -1)
    assert torch.all(c1 == -1).item()


@pytest.mark.parametrize("p", [1, 2, 3])
def test_quad_point_location_field_values(cuda, p):
    import torch
    from devil_ray_b200 import api
    from devil_ray_b200.render import PointLocation, QuadField
    m = _mesh(p)
    g = api.UnstructuredMesh(m.ctrl_idx, m.xyz, p, dim=2, device=cuda)
    f = QuadField(m.ctrl_idx, m.field, p, device=cuda)
    pts = _queries(20000, 20 + p)
    q = PointLocation()
    q.add_var("f")
    q.empty_val(-3.0)
    vals = q.execute(g, {"f": f}, pts)["f"].cpu().numpy()
    cell, rp = api.BatchedLocator(g, 1e-4, 20).locate(pts)
    torch.cuda.synchronize()
    cell, rp = cell.cpu().numpy(), rp.cpu().numpy()
    assert np.all(vals[cell < 0] == np.float32(-3.0))
    nd = (p + 1) ** 2
    conn = m.ctrl_idx.reshape(-1, nd)
    sel = np.nonzero(cell >= 0)[0][:4000]
    cv = m.field[conn[cell[sel]]].astype(np.float64).reshape(-1, p + 1, p + 1)   # [q, v, u]
    bu = _bern(p, rp[sel, 0].astype(np.float64))
    bv = _bern(p, rp[sel, 1].astype(np.float64))
    want = np.einsum("qvu,qu,qv->q", cv, bu, bv)
    assert np.abs(vals[sel] - want).max() < 1e-4
