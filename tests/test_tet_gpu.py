"""Tet (simplex) elements on the GPU, through the C-ABI, against the oracle.

  - sub-boxes (drb_elem_subboxes / drb_lbvh_build on a DRB_SHAPE_SIMPLEX
    mesh) bit-exact against the restated construct_bvh with the
    evaluators' dof layout at orders 1-3, and against the reference's own
    BVH (oracle/_ref) at order 1, where both layouts coincide;
  - point location (drb_locate, drb_locate_batched in both row modes)
    against the restated DeviceMesh::locate for tets over the same BVH, and
    against the reference's UnstructuredMesh<Tet> (general-order element
    type) at orders 1-2; order 3 is not run on the reference, whose order-3
    tet BVH build writes past its scratch array;
  - field values at located points (drb_field_eval) against the reference's
    Element<3,1,Simplex,General>::eval_d, and the forward map of located
    points (drb_map_points) back onto the queries.
Tolerances: cells identical on >= 99.9 % of queries (the rest must be valid
answers of the other side: the query maps into that element within 1e-4);
reference coordinates within 1e-4 of the FP32 oracle and 1e-3 of the
reference; field values within 1e-4.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ORDERS = [1, 2, 3]


def _mesh(p, n=6):
    from devil_ray_b200 import meshgen
    return meshgen.tet_warped_mesh(n, p, 0.05, jitter=0.01, seed=3 + p)


def _gpu(m, cuda):
    from devil_ray_b200 import _lib as L
    from devil_ray_b200 import api
    return api.UnstructuredMesh(m.ctrl_idx, m.xyz, m.order, device=cuda, shape=L.SHAPE_SIMPLEX)


def _bvh_np(b):
    return {"inner": b.inner_nodes.cpu().numpy(), "leaf_nodes": b.leaf_nodes.cpu().numpy(),
            "aabb_ids": b.aabb_ids.cpu().numpy(), "ref_boxes": b.ref_boxes.cpu().numpy()}


def _maps_back(g, cell, ref, pts, tol=1e-4):
    """The forward map X_cell(ref) of each located query lands on it."""
    import torch
    from devil_ray_b200.learned import map_points
    sel = cell >= 0
    X = map_points(g, torch.as_tensor(cell[sel], device=g.device),
                   torch.as_tensor(ref[sel], device=g.device)).cpu().numpy()
    return np.abs(X - pts[sel]).max(axis=1) < tol


@pytest.mark.parametrize("p", ORDERS)
def test_tet_subboxes_bit_exact(cuda, p):
    import torch
    from devil_ray_b200 import api
    from oracle import restate
    from tests.bvh_util import subbox_aabbs
    m = _mesh(p)
    g = _gpu(m, cuda)
    aabbs, prim, refb, bounds = api.elem_subboxes(g)
    b = g.build_bvh()
    torch.cuda.synchronize()
    a0, r0 = restate.tet_subboxes(p, m.ctrl_idx, m.xyz)
    assert np.array_equal(aabbs.cpu().numpy().view(np.int32), a0.view(np.int32))
    assert np.array_equal(refb.cpu().numpy().view(np.int32), r0.view(np.int32))
    assert np.array_equal(prim.cpu().numpy(), np.repeat(np.arange(m.n_elem, dtype=np.int32), 33))
    lo, hi = a0[:, 0::2].min(0), a0[:, 1::2].max(0)
    assert np.array_equal(bounds.cpu().numpy(), np.stack([lo, hi], 1).reshape(-1))
    # the built tree holds exactly these boxes, under their sub-box ids
    bn = _bvh_np(b)
    assert np.array_equal(subbox_aabbs(bn["inner"], bn["aabb_ids"]).view(np.int32), a0.view(np.int32))
    assert np.array_equal(bn["ref_boxes"].view(np.int32), r0.view(np.int32))


def test_tet_order1_bvh_matches_reference(cuda, ref):
    import torch
    from tests.bvh_util import subbox_aabbs
    m = _mesh(1)
    g = _gpu(m, cuda)
    b = g.build_bvh(keep_codes=True)
    torch.cuda.synchronize()
    rb = ref.RefTetMesh(1, m.ctrl_idx, m.xyz).bvh()
    bn = _bvh_np(b)
    ra = subbox_aabbs(rb["inner"], rb["aabb_ids"])
    assert np.array_equal(subbox_aabbs(bn["inner"], bn["aabb_ids"]).view(np.int32), ra.view(np.int32))
    assert np.array_equal(bn["ref_boxes"].view(np.int32), rb["ref_boxes"].view(np.int32))
    assert np.array_equal(b.bounds, rb["bounds"])
    codes, _ = ref.morton(ra)
    assert np.array_equal(np.sort(codes), b.sorted_codes.cpu().numpy().view(np.uint32))


@pytest.mark.parametrize("p", ORDERS)
@pytest.mark.parametrize("guess", ["zero", "elem_center", "subref_center"])
def test_tet_locate_matches_restated_oracle(cuda, p, guess):
    import torch
    from devil_ray_b200 import _lib as L
    from devil_ray_b200 import meshgen
    from oracle import restate
    mode = {"zero": L.GUESS_ZERO, "elem_center": L.GUESS_ELEM_CENTER,
            "subref_center": L.GUESS_SUBREF_CENTER}[guess]
    m = _mesh(p)
    g = _gpu(m, cuda)
    pts = meshgen.uniform_queries(40000, 17 + p)
    cell, rp = g.locate(pts, tol=1e-4, max_steps=20, guess_mode=mode)
    torch.cuda.synchronize()
    cell, rp = cell.cpu().numpy(), rp.cpu().numpy()
    oc, orf, _, _ = restate.locate_tet(p, m.ctrl_idx, m.xyz, _bvh_np(g.get_bvh()), pts, tol=1e-4,
                                       max_steps=20, guess_mode=mode, local_frame=True)
    same = cell == oc
    assert same.mean() > 0.999, f"{(~same).sum()} cell mismatches"
    both = same & (cell >= 0)
    assert np.abs(rp[both] - orf[both]).max() < 1e-4
    assert np.all(rp[cell < 0] == -1.0)
    assert 0.85 < (cell >= 0).mean() < 0.95
    assert _maps_back(g, cell, rp, pts).all()


@pytest.mark.parametrize("p", [1, 2])
def test_tet_locate_matches_reference(cuda, ref, p):
    import torch
    from devil_ray_b200 import _lib as L
    from devil_ray_b200 import meshgen
    m = _mesh(p)
    g = _gpu(m, cuda)
    pts = meshgen.uniform_queries(40000, 29 + p)
    cell, rp = g.locate(pts, tol=1e-4, max_steps=20, guess_mode=L.GUESS_ZERO)
    torch.cuda.synchronize()
    cell, rp = cell.cpu().numpy(), rp.cpu().numpy()
    rc, rr = ref.RefTetMesh(p, m.ctrl_idx, m.xyz).locate(pts)
    same = cell == rc
    assert same.mean() > 0.999, f"{(~same).sum()} cell mismatches"
    both = same & (cell >= 0)
    assert np.abs(rp[both] - rr[both]).max() < 1e-3
    # where the answers differ (order 2: the reference's boxes come from its
    # misindexed split, so candidates come in another order) ours is valid
    diff = ~same & (cell >= 0)
    if diff.any():
        assert _maps_back(g, np.where(diff, cell, -1), rp, pts).all()
    assert (cell >= 0).sum() >= (rc >= 0).sum()


@pytest.mark.parametrize("p", ORDERS)
@pytest.mark.parametrize("row_mode", [0, 1])
def test_tet_batched_identical_to_plain(cuda, p, row_mode):
    import torch
    from devil_ray_b200 import _lib as L
    from devil_ray_b200 import api, meshgen
    m = _mesh(p)
    g = _gpu(m, cuda)
    pts = meshgen.uniform_queries(60000, 41 + p)
    cell0, ref0 = g.locate(pts, tol=1e-5, max_steps=20, guess_mode=L.GUESS_ELEM_CENTER)
    cfg = L.DrbLocateConfig()
    cfg.block, cfg.blocks_per_sm, cfg.chunk, cfg.sort_queries, cfg.reg_elements = 128, 0, 64, 1, row_mode
    bl = api.BatchedLocator(g, tol=1e-5, max_steps=20, config=cfg)
    cell1, ref1 = bl.locate(pts)
    torch.cuda.synchronize()
    assert torch.equal(cell0, cell1)
    assert torch.equal(ref0.view(torch.int32), ref1.view(torch.int32))


@pytest.mark.parametrize("p", [1, 2])
def test_tet_face_neighbors(cuda, p):
    """Tet face-neighbour table against a NumPy restatement: face f of
    element e (u=0, v=0, w=0, u+v+w=1, by its three corner control points)
    and the other element with the same three corners; 2 (6 n^2) boundary
    faces on the n^3 x 6 Kuhn mesh."""
    import torch
    from devil_ray_b200 import meshgen
    n = 6
    m = _mesh(p, n)
    g = _gpu(m, cuda)
    nb = g.face_neighbors().cpu().numpy()
    torch.cuda.synchronize()
    nd = meshgen.tet_dofs(p)
    conn = np.asarray(m.ctrl_idx).reshape(-1, nd)
    # corner dofs of the (i, j, k) layout: u vertex (p,0,0), v vertex
    # (0,p,0), w vertex (0,0,p), origin (0,0,0)
    iv = sum(p + 1 - q for q in range(p))
    U, V, W, O = conn[:, p], conn[:, iv], conn[:, nd - 1], conn[:, 0]
    faces = [(V, W, O), (U, W, O), (U, V, O), (U, V, W)]
    owner = {}
    for f, cs in enumerate(faces):
        for e, key in enumerate(zip(*(np.sort(np.stack(cs, 1), axis=1).T))):
            owner.setdefault(key, []).append((e, f))
    want = np.full((conn.shape[0], 4), -1, np.int64)
    for key, lst in owner.items():
        assert len(lst) <= 2
        if len(lst) == 2:
            (a, fa), (b, fb) = lst
            want[a, fa], want[b, fb] = b, a
    assert nb.shape == (conn.shape[0], 4)
    assert np.array_equal(nb, want)
    assert (nb < 0).sum() == 2 * 6 * n * n


@pytest.mark.parametrize("p", ORDERS)
def test_tet_leaf_maps_match_fp64(cuda, p):
    """drb_bvh_leaf_maps on a tet mesh: each sampled leaf's record holds its
    sub-simplex centroid, the element map there and the inverse Jacobian,
    against an FP64 evaluation of the same element at the same point."""
    import torch
    from tests.bvh_util import leaf_maps_fp64
    m = _mesh(p)
    g = _gpu(m, cuda)
    b = g.get_bvh()
    b.build_leaf_maps(g)
    torch.cuda.synchronize()
    maps = b.leaf_maps.cpu().numpy()
    leaves = np.random.default_rng(5).choice(b.n_leaf, 3000, replace=False)
    want = leaf_maps_fp64("tet", p, m.ctrl_idx, m.xyz, b, leaves)
    got = maps[leaves, :15]
    assert np.array_equal(got[:, :3], want[:, :3].astype(np.float32))
    assert np.abs(got[:, 3:6] - want[:, 3:6]).max() < 1e-5
    scale = np.abs(want[:, 6:]).max(axis=1, keepdims=True)
    assert (np.abs(got[:, 6:] - want[:, 6:]) / scale).max() < 1e-4


@pytest.mark.parametrize("p", ORDERS)
def test_tet_subbox_linear_guess(cuda, p):
    """The first guess from each leaf's element map linearised at its
    sub-simplex centroid (GUESS_SUBBOX_LINEAR on a tet mesh) finds the same
    cells as the sub-simplex-centre guess (the rest: valid answers on shared
    faces), reference points within the 1e-5 tolerance, in fewer Newton
    steps; the plain and batched kernels agree bit for bit."""
    import torch
    from devil_ray_b200 import _lib as L
    from devil_ray_b200 import api, meshgen
    m = _mesh(p)
    g = _gpu(m, cuda)
    pts = meshgen.uniform_queries(60000, 53 + p)
    lin = api.BatchedLocator(g, tol=1e-5, max_steps=20, guess_mode=L.GUESS_SUBBOX_LINEAR)
    c4, r4, i4, _, _ = lin.locate(pts, stats=True)
    assert g.get_bvh().leaf_maps is not None
    cp, rp = g.locate(pts, tol=1e-5, max_steps=20, guess_mode=L.GUESS_SUBBOX_LINEAR)
    c2, r2, i2, *_ = api.BatchedLocator(g, 1e-5, 20, L.GUESS_SUBREF_CENTER).locate(pts, stats=True)
    torch.cuda.synchronize()
    assert torch.equal(c4, cp) and torch.equal(r4.view(torch.int32), rp.view(torch.int32))
    c4n, r4n, c2n, r2n = c4.cpu().numpy(), r4.cpu().numpy(), c2.cpu().numpy(), r2.cpu().numpy()
    same = c4n == c2n
    assert same.mean() > 0.999, f"{(~same).sum()} cell mismatches"
    assert _maps_back(g, np.where(~same, c4n, -1), r4n, pts).all()
    assert (c4n >= 0).sum() >= (c2n >= 0).sum() - 2
    both = same & (c4n >= 0)
    err = np.abs(r4n[both] - r2n[both]).max()
    loc = c4 >= 0
    m4, m2 = float(i4[loc].float().mean()), float(i2[loc].float().mean())
    print(f"tet p{p}: mean Newton steps: sub-simplex linear {m4:.3f}, centroid {m2:.3f}; "
          f"max ref diff {err:.2e}")
    assert err < 1e-5
    assert m4 < m2


@pytest.mark.parametrize("p", ORDERS)
def test_tet_point_location_field_values(cuda, ref, p):
    import torch
    from devil_ray_b200 import _lib as L
    from devil_ray_b200 import meshgen
    from devil_ray_b200.render import PointLocation, UnstructuredField
    from oracle import restate
    m = _mesh(p, n=4)
    g = _gpu(m, cuda)
    f = UnstructuredField(m.ctrl_idx, m.field, p, device=cuda, shape=L.SHAPE_SIMPLEX)
    pts = meshgen.uniform_queries(8000, 53 + p)
    q = PointLocation()
    q.add_var("f")
    q.empty_val(-7.0)
    vals = q.execute(g, {"f": f}, pts)["f"]
    from devil_ray_b200.api import BatchedLocator
    cell, rp = BatchedLocator(g, 1e-4, 20, L.GUESS_ELEM_CENTER).locate(pts)
    torch.cuda.synchronize()
    vals, cell, rp = vals.cpu().numpy(), cell.cpu().numpy(), rp.cpu().numpy()
    assert np.all(vals[cell < 0] == np.float32(-7.0))
    nd = meshgen.tet_dofs(p)
    conn = m.ctrl_idx.reshape(-1, nd)
    for e in np.unique(cell[cell >= 0])[:80]:
        sel = cell == e
        fv = m.field[conn[e]]
        X, _ = restate.tet_eval_d(p, fv.astype(np.float64), rp[sel].astype(np.float64))
        assert np.abs(vals[sel] - X[:, 0]).max() < 1e-4
        if p < 3:
            rv, _ = ref.eval_tet_scalar(p, fv, rp[sel])
            assert np.abs(vals[sel] - rv).max() < 1e-4


def test_face_neighbors_reject_2d_meshes(cuda):
    """Face tables are for hex and tet meshes: a 2D descriptor is rejected
    before anything is written."""
    import ctypes as C
    import torch
    from devil_ray_b200 import _lib as L
    m = _mesh(1, n=2)
    g = _gpu(m, cuda)
    d = g.desc()
    d.dim = 2
    buf = torch.full((4 * g.n_elem,), 7, dtype=torch.int32, device=cuda)
    st = L.lib().drb_mesh_face_neighbors(C.byref(d), C.c_void_p(buf.data_ptr()), None)
    assert st != 0
    assert "hex or tet" in L.lib().drb_last_error().decode()
    torch.cuda.synchronize()
    assert bool((buf == 7).all())


@pytest.mark.parametrize("p", [1, 2, 3])
def test_cpp_tet_mesh_interface(cuda, ref, tmp_path, p):
    """UnstructuredMesh<Tet*> / UnstructuredField<TetScalar*> through the C++
    host interface (t_dray_b200_tet): Mesh::locate against the restated
    oracle (and the reference at orders 1-2), PointLocation values against
    the element evaluation."""
    import subprocess
    from pathlib import Path
    from devil_ray_b200 import meshgen
    from oracle import restate
    exe = Path(__file__).resolve().parent.parent / "devil_ray_b200" / "cpp" / "tests" / "t_dray_b200_tet"
    if not exe.exists():
        pytest.fail("C++ test program missing: build with make -C devil_ray_b200/cpp")
    m = _mesh(p, n=5)
    pts = meshgen.uniform_queries(20000, 61 + p)
    with open(tmp_path / "mesh.bin", "wb") as f:
        np.array([p, m.n_elem, m.n_ctrl], np.int32).tofile(f)
        np.ascontiguousarray(m.ctrl_idx, np.int32).tofile(f)
        np.ascontiguousarray(m.xyz, np.float32).tofile(f)
        np.ascontiguousarray(m.field, np.float32).tofile(f)
    with open(tmp_path / "points.bin", "wb") as f:
        np.array([pts.shape[0]], np.int32).tofile(f)
        pts.tofile(f)
    from devil_ray_b200.render import Camera, PointLight
    cam_d = dict(pos=(2.5, 2.5, 2.5), look_at=(0.5, 0.5, 0.5), up=(0.0, 1.0, 0.0), fov=30.0)
    w, samples = 96, 300
    cam = Camera(w, w, cam_d["pos"], cam_d["look_at"], cam_d["up"], cam_d["fov"])
    light13 = PointLight.default(cam).as13()
    rgb = np.array(meshgen.TF_RGB, np.float32)
    alpha = np.array(meshgen.TF_ALPHA, np.float32)
    cam9 = np.array([*cam_d["pos"], *cam_d["look_at"], *cam_d["up"]], np.float32)
    with open(tmp_path / "render.bin", "wb") as f:
        np.array([w, w, samples], np.int32).tofile(f)
        np.array([*cam9, cam_d["fov"]], np.float32).tofile(f)
        np.asarray(light13, np.float32).reshape(13).tofile(f)
        np.array([rgb.shape[0]], np.int32).tofile(f)
        rgb.tofile(f)
        np.array([alpha.shape[0]], np.int32).tofile(f)
        alpha.tofile(f)
    r = subprocess.run([str(exe), str(tmp_path)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    n = pts.shape[0]
    raw = np.fromfile(tmp_path / "locate.bin", np.uint8)
    cell = raw[: 4 * n].view(np.int32)
    refp = raw[4 * n:].view(np.float32).reshape(n, 3)
    g = _gpu(m, cuda)
    oc, orf, _, _ = restate.locate_tet(p, m.ctrl_idx, m.xyz, _bvh_np(g.get_bvh()), pts, tol=1e-4,
                                       max_steps=20, guess_mode=0, local_frame=True)
    same = cell == oc
    assert same.mean() > 0.999
    assert np.abs(refp[same & (cell >= 0)] - orf[same & (cell >= 0)]).max() < 1e-4
    if p < 3:
        rc, _ = ref.RefTetMesh(p, m.ctrl_idx, m.xyz).locate(pts)
        assert (cell == rc).mean() > 0.999
    vals = np.fromfile(tmp_path / "pointloc.bin", np.float32)
    assert np.all(vals[cell < 0] == np.float32(-1e30))
    nd = meshgen.tet_dofs(p)
    conn = m.ctrl_idx.reshape(-1, nd)
    for e in np.unique(cell[cell >= 0])[:50]:
        sel = cell == e
        X, _ = restate.tet_eval_d(p, m.field[conn[e]].astype(np.float64), refp[sel].astype(np.float64))
        assert np.abs(vals[sel] - X[:, 0]).max() < 1e-4
    # Volume::integrate + composite over the tet mesh == the reference's image
    img = np.fromfile(tmp_path / "volume.bin", np.float32).reshape(w, w, 4)
    if p < 3:
        rimg, _ = ref.RefTetMesh(p, m.ctrl_idx, m.xyz, m.field).volume(
            w, w, cam9, cam_d["fov"], samples, True, 1024, rgb, alpha, light13[None])
        d = np.abs(img - rimg)
        assert np.any(d > 1.0 / 255.0, axis=-1).mean() < 0.005
    assert img[..., 3].max() > 0.1
    # MeshBoundary + Surface on the triangle faces; order 1 against the
    # reference's fixed-order tets (closed-form ray/triangle test)
    raw = np.fromfile(tmp_path / "surface.bin", np.float32)
    simg = raw[: 4 * w * w].reshape(w, w, 4)
    assert (simg[..., 3] > 0).mean() > 0.2
    if p == 1:
        rs = ref.RefTetMesh(1, m.ctrl_idx, m.xyz, m.field, fixed=True).surface(
            w, w, cam9, cam_d["fov"], 1024, rgb, alpha, light13[None])
        d = np.abs(simg - rs["rgba"])
        assert np.any(d > 1.0 / 255.0, axis=-1).mean() < 0.005


def _tet_volume(cuda, m, w, samples, lighting, coherent):
    import torch
    from devil_ray_b200 import _lib as L
    from devil_ray_b200 import meshgen
    from devil_ray_b200.render import Camera, ColorTable, PointLight, UnstructuredField, Volume
    c = dict(pos=(2.5, 2.5, 2.5), look_at=(0.5, 0.5, 0.5), up=(0.0, 1.0, 0.0), fov=30.0)
    cam = Camera(w, w, c["pos"], c["look_at"], c["up"], c["fov"])
    light = PointLight.default(cam)
    g = _gpu(m, cuda)
    f = UnstructuredField(m.ctrl_idx, m.field, m.order, device=cuda, shape=L.SHAPE_SIMPLEX)
    vol = Volume(g, f)
    vol.samples(samples)
    vol.use_lighting(lighting)
    t = ColorTable()
    for p in meshgen.TF_RGB:
        t.add_point(p[0], p[1:])
    for p in meshgen.TF_ALPHA:
        t.add_alpha(*p)
    vol.color_map().color_table(t)
    vol.color_map().samples(256)
    vol.coherent = coherent
    vol.guess_mode = L.GUESS_ZERO
    fb = vol.render(cam, [light])
    fb.composite_background()
    img = fb.image()
    torch.cuda.synchronize()
    cam9 = np.array([*c["pos"], *c["look_at"], *c["up"]], np.float32)
    return img, cam9, c["fov"], light


@pytest.mark.parametrize("p", [1, 2])
@pytest.mark.parametrize("coherent", [False, True])
def test_tet_volume_matches_reference(cuda, ref, p, coherent):
    """Volume::integrate + compositing over a tet mesh and field
    (dispatch_3d's TetMesh case) against the reference's image."""
    from devil_ray_b200 import meshgen
    m = _mesh(p, n=4)
    w, samples = 96, 300
    img, cam9, fov, light = _tet_volume(cuda, m, w, samples, True, coherent)
    rimg, _ = ref.RefTetMesh(p, m.ctrl_idx, m.xyz, m.field).volume(
        w, w, cam9, fov, samples, True, 256, np.array(meshgen.TF_RGB, np.float32),
        np.array(meshgen.TF_ALPHA, np.float32), light.as13()[None])
    d = np.abs(img - rimg)
    bad = np.any(d > 1.0 / 255.0, axis=-1)
    print(f"tet p{p} coherent={coherent}: max diff {d.max():.2e}, pixels > 1/255: {bad.sum()}")
    assert bad.mean() < 0.005
    assert (np.abs(rimg - rimg[0, 0]).max(-1) > 1e-3).mean() > 0.1   # the mesh covers the view


def test_tet_volume_order3_coherent_equals_plain(cuda):
    """Order 3 (not run on the reference): the coherent march (previous
    element first) and the plain per-sample BVH locate give the same image
    to within the Newton tolerance's effect on shading."""
    m = _mesh(3, n=4)
    a, _, _, _ = _tet_volume(cuda, m, 96, 300, True, False)
    b, _, _, _ = _tet_volume(cuda, m, 96, 300, True, True)
    d = np.abs(a - b)
    assert np.any(d > 1.0 / 255.0, axis=-1).mean() < 0.005
    assert (np.abs(a - a[0, 0]).max(-1) > 1e-3).mean() > 0.1


@pytest.mark.parametrize("p", ORDERS)
def test_tet_hull_filter_changes_nothing(cuda, p):
    """The batched locate's hull-plane filter (drb_tet_hull_planes) only
    skips solves that fail: results are bit-identical with and without it,
    with far fewer Newton steps; every control point is behind its planes."""
    import torch
    from devil_ray_b200 import _lib as L
    from devil_ray_b200 import api, meshgen
    m = _mesh(p)
    g = _gpu(m, cuda)
    g.get_bvh()
    hp = g.hull_planes().cpu().numpy().reshape(-1, 5, 4)
    nd = meshgen.tet_dofs(p)
    cps = m.xyz[m.ctrl_idx.reshape(-1, nd)].astype(np.float64)          # [n, nd, 3]
    side = np.einsum("efk,eik->efi", hp[:, :4, :3].astype(np.float64), cps) - hp[:, :4, 3:4]
    assert side.max() < 1e-6
    assert np.all(np.abs(np.linalg.norm(hp[:, :4, :3], axis=-1) - 1.0) < 1e-5)
    pts = meshgen.uniform_queries(60000, 71 + p)
    bl = api.BatchedLocator(g, tol=1e-5, max_steps=20)
    c1, r1, it1, ca1, _ = bl.locate(pts, stats=True)
    saved, g._hull = g._hull, None
    try:
        c0, r0, it0, ca0, _ = bl.locate(pts, stats=True)
    finally:
        g._hull = saved
    torch.cuda.synchronize()
    assert torch.equal(c0, c1)
    assert torch.equal(r0.view(torch.int32), r1.view(torch.int32))
    assert torch.equal(ca0, ca1)
    assert it1.sum().item() < 0.6 * it0.sum().item()


def _tet_surface(cuda, m, w):
    import torch
    from devil_ray_b200 import _lib as L
    from devil_ray_b200 import meshgen
    from devil_ray_b200.render import (Camera, ColorTable, MeshBoundary, PointLight, Surface,
                                       UnstructuredField)
    c = dict(pos=(2.5, 2.5, 2.5), look_at=(0.5, 0.5, 0.5), up=(0.0, 1.0, 0.0), fov=30.0)
    cam = Camera(w, w, c["pos"], c["look_at"], c["up"], c["fov"])
    light = PointLight.default(cam)
    g = _gpu(m, cuda)
    f = UnstructuredField(m.ctrl_idx, m.field, m.order, device=cuda, shape=L.SHAPE_SIMPLEX)
    mb = MeshBoundary()
    faces, ff = mb.execute(g, f)
    surf = Surface(faces, ff)
    t = ColorTable()
    for p in meshgen.TF_RGB:
        t.add_point(p[0], p[1:])
    for p in meshgen.TF_ALPHA:
        t.add_alpha(*p)
    surf.color_map().color_table(t)
    fb, hits = surf.render(cam, [light])
    torch.cuda.synchronize()
    cam9 = np.array([*c["pos"], *c["look_at"], *c["up"]], np.float32)
    return g, faces, fb, hits, cam, cam9, c["fov"], light


@pytest.mark.parametrize("p", [1, 2, 3])
def test_tet_boundary_faces(cuda, ref, p):
    """MeshBoundary on a tet mesh: 2 triangles per boundary square; at order
    1 the face list is the reference's (same order, same vertex order)."""
    import torch
    from devil_ray_b200 import _lib as L
    from devil_ray_b200.render import MeshBoundary
    m = _mesh(p, n=3)
    g = _gpu(m, cuda)
    faces, _ = MeshBoundary().execute(g)
    torch.cuda.synchronize()
    fi = faces.dof_data.ctrl_idx.cpu().numpy().reshape(faces.n_elem, -1)
    assert fi.shape == (6 * 2 * 9, (p + 1) * (p + 2) // 2)
    assert faces.shape == L.SHAPE_SIMPLEX and faces.dim == 2
    # every face dof lies on the cube's boundary (lattice coordinate 0 or max)
    mm = p * 3 + 1
    K, r = np.divmod(fi, mm * mm)
    J, I = np.divmod(r, mm)
    on = (I == 0) | (I == mm - 1) | (J == 0) | (J == mm - 1) | (K == 0) | (K == mm - 1)
    assert on.all()
    if p == 1:
        rb = ref.RefTetMesh(1, m.ctrl_idx, m.xyz, fixed=True).boundary_ctrl_idx()
        assert np.array_equal(fi, rb)


def test_tet_surface_order1_matches_reference(cuda, ref):
    """Triangle faces of order-1 tets through the closed-form ray/triangle
    test (FaceIntersector<Tri_P1>, restated operation for operation): hits,
    distances and (u, v) bit for bit; image within 1/255."""
    from devil_ray_b200 import meshgen
    m = _mesh(1, n=5)
    w = 128
    g, faces, fb, hits, cam, cam9, fov, light = _tet_surface(cuda, m, w)
    rs = ref.RefTetMesh(1, m.ctrl_idx, m.xyz, m.field, fixed=True).surface(
        w, w, cam9, fov, 1024, np.array(meshgen.TF_RGB, np.float32),
        np.array(meshgen.TF_ALPHA, np.float32), light.as13()[None])
    h = hits.cpu().numpy()
    gidx = h[:, 0].view(np.int32)
    same = gidx == rs["hit_idx"]
    assert same.mean() > 0.998, f"{(~same).sum()} hit mismatches"
    both = same & (gidx >= 0)
    assert both.mean() > 0.2
    assert np.array_equal(h[both, 1].view(np.int32), rs["dist"][both].view(np.int32))
    assert np.array_equal(h[both, 2:4].view(np.int32), rs["ref"][both].view(np.int32))
    d = np.abs(fb.image() - rs["rgba"])
    assert np.any(d > 1.0 / 255.0, axis=-1).mean() < 0.005


@pytest.mark.parametrize("p", [2, 3])
def test_tet_surface_curved_faces_lie_on_rays(cuda, p):
    """Curved triangle faces (Newton ray/face solve): every hit's face point
    X(u, v) is the ray's point at the hit distance, (u, v) lies in the
    triangle, and a query just past the hit is located inside the tet mesh
    while one just before it is not (the face is the mesh's boundary)."""
    import torch
    from math import factorial
    from devil_ray_b200 import meshgen
    m = _mesh(p, n=5)
    w = 128
    g, faces, fb, hits, cam, cam9, fov, light = _tet_surface(cuda, m, w)
    h = hits.cpu().numpy()
    gidx = h[:, 0].view(np.int32)
    sel = np.nonzero(gidx >= 0)[0]
    assert sel.size > 0.2 * w * w
    rays = cam.create_rays(cuda).cpu().numpy()
    orig, dirs = rays[sel, 4:7].astype(np.float64), rays[sel, 0:3].astype(np.float64)
    tdist = h[sel, 1].astype(np.float64)
    u, v = h[sel, 2].astype(np.float64), h[sel, 3].astype(np.float64)
    fi = faces.dof_data.ctrl_idx.cpu().numpy().reshape(faces.n_elem, -1)
    cp = m.xyz[fi[gidx[sel]]].astype(np.float64)                 # [k, nd2, 3]
    t = 1 - u - v
    X = np.zeros((sel.size, 3))
    for j in range(p + 1):
        for i in range(p + 1 - j):
            l = p - i - j
            B = factorial(p) / (factorial(i) * factorial(j) * factorial(l)) * u ** i * v ** j * t ** l
            X += B[:, None] * cp[:, (2 * p + 3 - j) * j // 2 + i]
    on_ray = orig + tdist[:, None] * dirs
    assert np.abs(X - on_ray).max() < 2e-4
    assert (np.minimum(np.minimum(u, v), t) >= -1.1e-4).all()
    eps = 2e-3
    q_in = torch.as_tensor((on_ray + eps * dirs).astype(np.float32), device=cuda)
    q_out = torch.as_tensor((on_ray - eps * dirs).astype(np.float32), device=cuda)
    from devil_ray_b200 import api
    c_in, _ = api.BatchedLocator(g).locate(q_in)
    c_out, _ = api.BatchedLocator(g).locate(q_out)
    torch.cuda.synchronize()
    assert (c_in >= 0).float().mean().item() > 0.98
    assert (c_out < 0).float().mean().item() > 0.98


@pytest.mark.parametrize("p", ORDERS)
@pytest.mark.parametrize("guess", ["zero", "center", "subref"])
def test_tet_batched_skips_only_failing_solves(cuda, p, guess):
    """The batched locate skips a candidate tet whose solve already failed
    for the query (leaf-independent guesses) and tets whose hull planes
    reject the query. Against the plain kernel, which solves every
    candidate: the same cells and reference points bit for bit, the same
    candidate counts, and never more Newton steps for any query."""
    import torch
    from devil_ray_b200 import _lib as L
    from devil_ray_b200 import api, meshgen
    m = _mesh(p)
    g = _gpu(m, cuda)
    mode = {"zero": L.GUESS_ZERO, "center": L.GUESS_ELEM_CENTER,
            "subref": L.GUESS_SUBREF_CENTER}[guess]
    pts = torch.as_tensor(meshgen.uniform_queries(60000, 91 + p), device=cuda)
    c0, r0, it0, ca0, _ = g.locate(pts, tol=1e-5, max_steps=20, guess_mode=mode, stats=True)
    bl = api.BatchedLocator(g, tol=1e-5, max_steps=20, guess_mode=mode)
    c1, r1, it1, ca1, _ = bl.locate(pts, stats=True)
    torch.cuda.synchronize()
    assert torch.equal(c0, c1)
    assert torch.equal(r0.view(torch.int32), r1.view(torch.int32))
    assert torch.equal(ca0, ca1)
    assert bool((it1 <= it0).all())
    if guess != "subref":
        assert it1.sum().item() < it0.sum().item()
