"""Rendering parity on the GPU against the reference (oracle/_ref):
camera rays bit-exact, volume images within 1/255 per channel."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CAM = dict(pos=(2.5, 2.5, 2.5), look_at=(0.5, 0.5, 0.5), up=(0.0, 1.0, 0.0), fov=30.0)


def cam9():
    return np.array([*CAM["pos"], *CAM["look_at"], *CAM["up"]], np.float32)


@pytest.mark.parametrize("wh", [(256, 256), (300, 200), (64, 97)])
def test_camera_rays_bit_exact(cuda, ref, wh):
    from devil_ray_b200.render import Camera
    w, h = wh
    rr = ref.camera_rays(w, h, cam9(), CAM["fov"])
    c = Camera(w, h, CAM["pos"], CAM["look_at"], CAM["up"], CAM["fov"])
    g = c.create_rays(cuda).cpu().numpy()
    assert np.array_equal(g.view(np.uint32), rr.view(np.uint32))


def _mesh(name):
    """volume_8, or p3_N: the order-3 warped mesh family of the 128^3 volume
    workload at N^3 elements."""
    from devil_ray_b200 import meshgen
    if name.startswith("p3_"):
        return meshgen.warped_mesh(int(name[3:]), 3, 0.05, gaussian_field_seed=4)
    return meshgen.workload_mesh(name)


def _volume_case(cuda, ref, mesh_name, w, samples, lighting, coherent, guess):
    import torch
    from devil_ray_b200 import _lib as L
    from devil_ray_b200 import api, meshgen
    from devil_ray_b200.render import Camera, ColorTable, PointLight, UnstructuredField, Volume
    m = _mesh(mesh_name)
    cam = Camera(w, w, CAM["pos"], CAM["look_at"], CAM["up"], CAM["fov"])
    light = PointLight.default(cam)
    rgb = np.array(meshgen.TF_RGB, np.float32)
    alpha = np.array(meshgen.TF_ALPHA, np.float32)
    r = ref.RefHexMesh(m.order, m.ctrl_idx, m.xyz, m.field)
    rimg, rparts = r.volume(w, w, cam9(), CAM["fov"], samples, lighting, 256, rgb, alpha,
                            light.as13()[None], want_partials=True)
    mesh = api.UnstructuredMesh(m.ctrl_idx, m.xyz, m.order, device=cuda)
    field = UnstructuredField(m.ctrl_idx, m.field, m.order, device=cuda)
    vol = Volume(mesh, field)
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
    vol.guess_mode = guess
    fb = vol.render(cam, [light])
    fb.composite_background()
    img = fb.image()
    parts = vol.integrate(cam.create_rays(cuda), [light])
    torch.cuda.synchronize()
    return rimg, rparts, img, parts


def _near_face_rays(cuda, ref, m, w, samples, pixels, band=2e-4):
    """For each pixel, whether its ray has a sample point on an element
    face: one that the reference's locate or the GPU's puts within `band`
    of a face of its element (a face shared by two elements, which either
    may own within the Newton tolerance), or one just outside the mesh that
    the reference misses while Newton accepts it within the tolerance in the
    element of the ray's previous sample (the coherent march tries that
    element first; a BVH locate never considers a point outside every
    leaf box).  The sample points are the reference march's:
    near + k * dt with dt = |bounds diagonal| / samples, accumulated in
    float32 (rendering/volume.cpp:89-99,148-205)."""
    import torch
    from devil_ray_b200 import api
    from devil_ray_b200.render import Camera, cull_rays
    g = api.UnstructuredMesh(m.ctrl_idx, m.xyz, m.order, device=cuda)
    b = g.bounds()
    cam = Camera(w, w, CAM["pos"], CAM["look_at"], CAM["up"], CAM["fov"])
    active = cull_rays(cam.create_rays(cuda), b).cpu().numpy()
    pid = active[:, 8].view(np.int32)
    lo = np.array(b[0::2], np.float32)
    hi = np.array(b[1::2], np.float32)
    e = (hi - lo).astype(np.float32)
    mag = np.sqrt(np.float32(e[0] * e[0] + e[1] * e[1] + e[2] * e[2]), dtype=np.float32)
    dt = np.float32(mag / np.float32(samples))
    rm = ref.RefHexMesh(m.order, m.ctrl_idx, m.xyz)
    from devil_ray_b200 import _lib as L
    out = np.zeros(len(pixels), bool)
    for k, px in enumerate(pixels):
        sel = np.nonzero(pid == px)[0]
        if sel.size == 0:
            continue
        r = active[sel[0]]
        d = np.float32(r[3]) + dt
        pts = []
        while d < np.float32(r[7]):
            pts.append(r[4:7] + d * r[0:3])
            d = np.float32(d + dt)
        if not pts:
            continue
        pts = np.asarray(pts, np.float32)
        cell, rr = rm.locate(pts)
        gc, gr = g.locate(pts, tol=1e-4, max_steps=20, guess_mode=L.GUESS_ZERO)
        gc, gr = gc.cpu().numpy(), gr.cpu().numpy()
        ins = np.concatenate([rr[cell >= 0], gr[gc >= 0]])
        out[k] = bool(np.any((ins < band) | (ins > 1.0 - band)))
        if not out[k]:
            # exits: a missed sample after a located one, solved in that element
            j = np.nonzero((cell[1:] < 0) & (cell[:-1] >= 0))[0] + 1
            if j.size:
                from devil_ray_b200.learned import newton_pairs
                el = torch.as_tensor(cell[j - 1], dtype=torch.int32, device=cuda)
                p = torch.as_tensor(pts[j], device=cuda)
                x, _, _ = newton_pairs(g, el, p, 1e-5, 20)
                x = x.cpu().numpy()
                out[k] = bool(np.any(np.all((x > -band) & (x < 1.0 + band), axis=1)))
    return out


@pytest.mark.parametrize("coherent", [0, 1, 2])
@pytest.mark.parametrize("lighting", [True, False])
def test_volume_image_matches_reference(cuda, ref, coherent, lighting):
    """Images within 1/255 per channel, except pixels whose ray samples a
    point on a face shared by two elements: there the element that owns the
    sample may differ, and with lighting so does the field gradient (the
    field is only continuous across faces).  Every such pixel is checked to
    be one of those rays."""
    from devil_ray_b200 import _lib as L
    from devil_ray_b200 import meshgen
    w, samples = 128, 500
    rimg, rparts, img, parts = _volume_case(cuda, ref, "volume_8", w, samples, lighting,
                                            coherent, L.GUESS_ZERO)
    d = np.abs(img - rimg)
    bad = np.any(d > 1.0 / 255.0, axis=-1)
    print(f"coherent={coherent} lighting={lighting}: max diff {d.max():.2e}, "
          f"pixels > 1/255: {bad.sum()} of {bad.size}; partials {parts.shape[0]} vs {len(rparts)}")
    assert bad.mean() < 0.002
    assert d.max() < 0.05
    assert abs(parts.shape[0] - len(rparts)) <= max(2, 0.002 * len(rparts))
    pixels = np.nonzero(bad.ravel())[0]
    if pixels.size:
        on_face = _near_face_rays(cuda, ref, meshgen.workload_mesh("volume_8"), w, samples,
                                  pixels)
        print(f"  of those, rays through a shared face: {on_face.sum()}")
        assert on_face.all(), f"pixels {pixels[~on_face]} differ without a shared-face sample"


def test_volume_partials_match_reference(cuda, ref):
    from devil_ray_b200 import _lib as L
    rimg, rparts, img, parts = _volume_case(cuda, ref, "volume_8", 96, 200, True, False,
                                            L.GUESS_ZERO)
    p = parts.cpu().numpy()
    pix = p[:, 0].view(np.int32)
    rpix = rparts[:, 0].astype(np.int32)
    # the same segments: counts equal, and per pixel the same number of
    # partials (a shared-face sample may split or join a segment: at most a
    # few pixels differ)
    assert abs(len(pix) - len(rpix)) <= max(2, 0.002 * len(rpix))
    cnt = np.bincount(pix, minlength=96 * 96)
    rcnt = np.bincount(rpix, minlength=96 * 96)
    assert (cnt != rcnt).mean() < 0.002
    # pixels with the same segments: depths bit-equal in the main, colours close
    same_pix = np.nonzero(cnt == rcnt)[0]
    keep = np.isin(pix, same_pix)
    rkeep = np.isin(rpix, same_pix)
    a, b = p[keep], rparts[rkeep]
    assert np.array_equal(a[:, 0].view(np.int32), b[:, 0].astype(np.int32))
    dd = np.abs(a[:, 1] - b[:, 1])
    assert np.median(dd) == 0.0
    assert np.abs(a[:, 2:] - b[:, 2:]).max() < 0.05


@pytest.mark.parametrize("name,w,samples", [("p3_6", 96, 300), ("p3_24", 192, 1000)])
def test_volume_order3(cuda, ref, name, w, samples):
    """Order 3, the volume workload's mesh family (at 24^3 the workload's
    1000 samples), lit, through the coherent march with the quadratic
    predictor and the face walk: within 1/255 per channel except rays
    through a shared face, each of which is checked to be one."""
    from devil_ray_b200 import _lib as L
    rimg, rparts, img, parts = _volume_case(cuda, ref, name, w, samples, True, 2, L.GUESS_ZERO)
    d = np.abs(img - rimg)
    bad = np.any(d > 1.0 / 255.0, axis=-1)
    print(f"{name}: max diff {d.max():.2e}, pixels > 1/255: {bad.sum()} of {bad.size}")
    assert bad.mean() < 0.005
    pixels = np.nonzero(bad.ravel())[0]
    if pixels.size:
        on_face = _near_face_rays(cuda, ref, _mesh(name), w, samples, pixels)
        print(f"  of those, rays through a shared face: {on_face.sum()}")
        assert on_face.all(), f"pixels {pixels[~on_face]} differ without a shared-face sample"


def test_volume_wide_traversal_identical(cuda):
    """The march's full locates over the 4-wide tree give the same image,
    bit for bit, as over the binary tree (plain and coherent)."""
    import torch
    from devil_ray_b200 import api, meshgen
    from devil_ray_b200.render import Camera, ColorTable, PointLight, UnstructuredField, Volume
    m = meshgen.warped_mesh(6, 3, 0.05, gaussian_field_seed=4)
    g = api.UnstructuredMesh(m.ctrl_idx, m.xyz, m.order, device=cuda)
    gb = api.UnstructuredMesh(m.ctrl_idx, m.xyz, m.order, device=cuda)
    gb._bvh = g.get_bvh().binary_only()
    assert g.get_bvh().wide_nodes is not None and gb.get_bvh().wide_nodes is None
    field = UnstructuredField(m.ctrl_idx, m.field, m.order, device=cuda)
    cam = Camera(96, 96, CAM["pos"], CAM["look_at"], CAM["up"], CAM["fov"])
    light = PointLight.default(cam)
    imgs = []
    for coherent in (False, True):
        for mesh in (g, gb):
            vol = Volume(mesh, field)
            vol.samples(300)
            t = ColorTable()
            for p in meshgen.TF_RGB:
                t.add_point(p[0], p[1:])
            for p in meshgen.TF_ALPHA:
                t.add_alpha(*p)
            vol.color_map().color_table(t)
            vol.coherent = coherent
            fb = vol.render(cam, [light])
            torch.cuda.synchronize()
            imgs.append(fb.image())
    assert np.array_equal(imgs[0].view(np.int32), imgs[1].view(np.int32))
    assert np.array_equal(imgs[2].view(np.int32), imgs[3].view(np.int32))


def test_face_neighbors(cuda):
    """Face-neighbour table: 6 n^2 boundary faces on an n^3 mesh, and every
    neighbour across face f shares that face's four corners as its own
    opposite face (the lattice keeps the axes)."""
    import torch
    from devil_ray_b200 import api, meshgen
    n, p = 5, 3
    m = meshgen.warped_mesh(n, p, 0.05)
    g = api.UnstructuredMesh(m.ctrl_idx, m.xyz, m.order, device=cuda)
    nb = g.face_neighbors().cpu().numpy()
    torch.cuda.synchronize()
    assert nb.shape == (n ** 3, 6)
    assert (nb < 0).sum() == 6 * n * n
    conn = np.asarray(m.ctrl_idx).reshape(-1, (p + 1) ** 3)
    n1 = p + 1

    def corners(e, f):
        axis, side = f // 2, (f % 2) * p
        out = []
        for s in (0, p):
            for r in (0, p):
                abc = [0, 0, 0]
                abc[axis], abc[(axis + 1) % 3], abc[(axis + 2) % 3] = side, s, r
                out.append(conn[e, (abc[2] * n1 + abc[1]) * n1 + abc[0]])
        return sorted(out)

    for e in range(n ** 3):
        for f in range(6):
            o = nb[e, f]
            if o >= 0:
                assert o != e and nb[o, f ^ 1] == e
                assert corners(e, f) == corners(o, f ^ 1)
