"""Non-synthetic inputs on the GPU: the reference's own order-1 MFEM test
meshes (beam-hex, fichera, beam-tet and the 2D beam-quad, beam-tri), read by
devil_ray_b200.mesh_io into the committed fixture arrays, through the path
against the reference itself (oracle/_ref) given the same arrays:

* point location at the reference's settings: cells identical except for
  points on faces shared by two elements, reference points within 1e-5;
* the boundary faces and the surface render (order-1 faces are intersected
  in closed form, so hits, distances and (u, v) are bit-exact);
* the volume render of a vertex field, within 1/255 per channel.
"""
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIXTURE = Path(__file__).resolve().parent / "golden" / "mfem_order1_meshes.npz"


def _load(name):
    from devil_ray_b200 import mesh_io
    fx = np.load(FIXTURE)
    shape = str(fx[f"{name}/shape"])
    m = mesh_io.LowOrderMesh(shape, fx[f"{name}/ctrl_idx"], fx[f"{name}/xyz"], 1, name)
    x, y, z = (m.xyz[:, k].astype(np.float64) for k in range(3))
    field = (np.sin(3 * x) * np.cos(2 * y) + z ** 2).astype(np.float32)
    return m, field


def _ref_mesh(ref, m, field=None, fixed_tets=False):
    """The reference mesh over the same arrays.  Tets: the general-order
    element type (its fixed order-1 type writes all three derivatives into
    the first Jacobian column, so its locate fails); the surface test takes
    the fixed type, whose face intersection does not use that evaluation."""
    cls = {"hex": ref.RefHexMesh, "tet": ref.RefTetMesh, "quad": ref.RefQuadMesh,
           "tri": ref.RefTriMesh}[m.shape]
    if m.shape == "tet":
        return cls(1, m.ctrl_idx, m.xyz, field, fixed=fixed_tets)
    return cls(1, m.ctrl_idx, m.xyz, field)


def _queries(m, n, seed):
    lo, hi = m.xyz.min(0), m.xyz.max(0)
    pad = 0.05 * (hi - lo)
    q = np.random.default_rng(seed).uniform(lo - pad, hi + pad, size=(n, 3)).astype(np.float32)
    if m.dim == 2:
        q[:, 2] = 0.0
    return q


def _camera(m, w):
    """A camera that frames the mesh: looking at the bounds' centre from
    a direction (1, 0.8, 1.4) at 1.8 times the bounds' diagonal."""
    from devil_ray_b200.render import Camera
    lo, hi = m.xyz.min(0).astype(np.float64), m.xyz.max(0).astype(np.float64)
    c = 0.5 * (lo + hi)
    d = np.array([1.0, 0.8, 1.4])
    d /= np.linalg.norm(d)
    pos = c + 1.8 * np.linalg.norm(hi - lo) * d
    cam = Camera(w, w, tuple(float(v) for v in pos), tuple(float(v) for v in c),
                 (0.0, 1.0, 0.0), 30.0)
    cam9 = np.array([*pos, *c, 0.0, 1.0, 0.0], np.float32)
    return cam, cam9


def _on_shared_face(m, cell_a, ref_a, band=2e-3):
    """The answer lies on the boundary band of its element."""
    if m.simplex:
        bary = np.concatenate([ref_a[:, :m.dim], 1.0 - ref_a[:, :m.dim].sum(1, keepdims=True)], 1)
        return np.any(bary < band, axis=1)
    r = ref_a[:, :m.dim]
    return np.any((r < band) | (r > 1.0 - band), axis=1)


@pytest.mark.parametrize("name", ["beam-hex", "fichera", "beam-tet", "beam-quad", "beam-tri"])
def test_imported_mesh_locate_matches_reference(cuda, ref, name):
    import torch
    from devil_ray_b200 import _lib as L
    m, _ = _load(name)
    q = _queries(m, 60000, 41)
    rc, rr = _ref_mesh(ref, m).locate(q)
    g = m.device_mesh(cuda)
    cell, rf = g.locate(q, tol=1e-4, max_steps=20, guess_mode=L.GUESS_ZERO)
    torch.cuda.synchronize()
    cell, rf = cell.cpu().numpy(), rf.cpu().numpy()
    same = cell == rc
    diff = ~same
    both_found = diff & (cell >= 0) & (rc >= 0)
    assert _on_shared_face(m, cell[both_found], rf[both_found]).all()
    assert _on_shared_face(m, rc[both_found], rr[both_found]).all()
    assert diff.mean() < 2e-3, f"{name}: {diff.sum()} cell mismatches"
    hit = same & (cell >= 0)
    assert hit.mean() > 0.3
    err = np.abs(rf[hit][:, :m.dim] - rr[hit][:, :m.dim]).max()
    print(f"{name}: {m.n_elem} {m.shape}, located {np.mean(cell >= 0):.3f}, "
          f"mismatches {diff.sum()}, max ref diff {err:.2e}")
    assert err < 1e-5


@pytest.mark.parametrize("name", ["beam-hex", "fichera", "beam-tet"])
def test_imported_mesh_surface_matches_reference(cuda, ref, name):
    import torch
    from devil_ray_b200 import _lib as L
    from devil_ray_b200 import meshgen
    from devil_ray_b200.render import (ColorTable, MeshBoundary, PointLight, Surface,
                                       UnstructuredField)
    m, field = _load(name)
    r = _ref_mesh(ref, m, field, fixed_tets=True)
    g = m.device_mesh(cuda)
    shape = L.SHAPE_SIMPLEX if m.simplex else L.SHAPE_TENSOR
    f = UnstructuredField(m.ctrl_idx, field, 1, device=cuda, shape=shape)
    faces, ff = MeshBoundary().execute(g, f)
    gfaces = faces.dof_data.ctrl_idx.cpu().numpy().reshape(faces.n_elem, -1)
    assert np.array_equal(gfaces, r.boundary_ctrl_idx().reshape(gfaces.shape[0], -1))
    w = 192
    cam, cam9 = _camera(m, w)
    light = PointLight.default(cam)
    surf = Surface(faces, ff)
    t = ColorTable()
    for p in meshgen.TF_RGB:
        t.add_point(p[0], p[1:])
    for p in meshgen.TF_ALPHA:
        t.add_alpha(*p)
    surf.color_map().color_table(t)
    fb, hits = surf.render(cam, [light])
    torch.cuda.synchronize()
    rs = r.surface(w, w, cam9, 30.0, 1024, np.array(meshgen.TF_RGB, np.float32),
                   np.array(meshgen.TF_ALPHA, np.float32), light.as13()[None])
    h = hits.cpu().numpy()
    gidx = h[:, 0].view(np.int32)
    same = gidx == rs["hit_idx"]
    both = same & (gidx >= 0)
    assert both.mean() > 0.1
    assert same.mean() > 0.995, f"{(~same).sum()} hit mismatches"
    assert np.array_equal(h[both, 1].view(np.int32), rs["dist"][both].view(np.int32))
    assert np.array_equal(h[both, 2:4].view(np.int32), rs["ref"][both].view(np.int32))
    d = np.abs(fb.image() - rs["rgba"])
    bad = np.any(d > 1.0 / 255.0, axis=-1)
    print(f"{name}: hits {np.mean(gidx >= 0):.3f}, mismatched hits {(~same).sum()}, "
          f"pixels > 1/255: {bad.sum()}")
    # every pixel over the bar is a ray whose hit differs (a shared edge)
    assert not np.any(bad.ravel() & same)


@pytest.mark.parametrize("name", ["beam-hex", "fichera"])
def test_imported_mesh_volume_matches_reference(cuda, ref, name):
    import torch
    from devil_ray_b200 import _lib as L
    from devil_ray_b200 import meshgen
    from devil_ray_b200.render import ColorTable, PointLight, UnstructuredField, Volume
    m, field = _load(name)
    w = 128
    cam, cam9 = _camera(m, w)
    light = PointLight.default(cam)
    r = _ref_mesh(ref, m, field)
    rimg, _ = r.volume(w, w, cam9, 30.0, 400, True, 256, np.array(meshgen.TF_RGB, np.float32),
                       np.array(meshgen.TF_ALPHA, np.float32), light.as13()[None])
    g = m.device_mesh(cuda)
    f = UnstructuredField(m.ctrl_idx, field, 1, device=cuda)
    vol = Volume(g, f)
    vol.samples(400)
    vol.use_lighting(True)
    t = ColorTable()
    for p in meshgen.TF_RGB:
        t.add_point(p[0], p[1:])
    for p in meshgen.TF_ALPHA:
        t.add_alpha(*p)
    vol.color_map().color_table(t)
    vol.color_map().samples(256)
    vol.guess_mode = L.GUESS_ZERO
    fb = vol.render(cam, [light])
    fb.composite_background()
    img = fb.image()
    torch.cuda.synchronize()
    d = np.abs(img - rimg)
    bad = np.any(d > 1.0 / 255.0, axis=-1)
    print(f"{name}: max diff {d.max():.2e}, pixels > 1/255: {bad.sum()} of {bad.size}")
    assert bad.mean() < 0.002


@pytest.mark.parametrize("name", ["beam-hex", "fichera", "beam-tet", "beam-quad", "beam-tri"])
@pytest.mark.parametrize("scale", [0.5, 1.0])
def test_imported_mesh_grid_locate_equals_plain(cuda, name, scale):
    """On the reference's own meshes (irregular element sizes, a re-entrant
    corner in fichera), the batched locate over grid candidate lists gives
    the plain kernel's answers bit for bit at the reference's settings."""
    import torch
    from devil_ray_b200 import _lib as L
    from devil_ray_b200 import api
    m, _ = _load(name)
    q = _queries(m, 40000, 43)
    g = m.device_mesh(cuda)
    c0, r0 = g.locate(q, tol=1e-4, max_steps=20, guess_mode=L.GUESS_ZERO)
    grid = g.get_bvh().without_grid().build_grid(scale)
    c1, r1 = api.BatchedLocator(g, tol=1e-4, max_steps=20, guess_mode=L.GUESS_ZERO,
                                bvh=grid).locate(q)
    torch.cuda.synchronize()
    assert torch.equal(c0, c1)
    assert torch.equal(r0.view(torch.int32), r1.view(torch.int32))
    assert (c1 >= 0).float().mean() > 0.3
