"""The C++ host interface (libdray_b200.so, namespace dray) against the
reference: the test program devil_ray_b200/cpp/tests/t_dray_b200_path runs
Mesh::locate, PointLocation, Volume::integrate + composite and
MeshBoundary + Surface through the C++ classes a reference user calls, and
this file compares its outputs with the same calls made on the reference
(oracle/_ref)."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
EXE = ROOT / "devil_ray_b200" / "cpp" / "tests" / "t_dray_b200_path"
CAM = dict(pos=(2.5, 2.5, 2.5), look_at=(0.5, 0.5, 0.5), up=(0.0, 1.0, 0.0), fov=30.0)


def test_cpp_library_loads():
    """libdray_b200.so resolves against libdrb.so without a GPU."""
    import ctypes
    so = ROOT / "devil_ray_b200" / "libdray_b200.so"
    if not so.exists():
        pytest.skip("C++ interface not built (make -C devil_ray_b200/cpp)")
    ctypes.CDLL(str(so))
    assert EXE.exists()


def _write_inputs(d, m, pts, w, samples, light13):
    with open(d / "mesh.bin", "wb") as f:
        np.array([m.order, m.ctrl_idx.size // (m.order + 1) ** 3, m.xyz.shape[0]],
                 np.int32).tofile(f)
        np.ascontiguousarray(m.ctrl_idx, np.int32).tofile(f)
        np.ascontiguousarray(m.xyz, np.float32).tofile(f)
        np.ascontiguousarray(m.field, np.float32).tofile(f)
    with open(d / "points.bin", "wb") as f:
        np.array([pts.shape[0]], np.int32).tofile(f)
        np.ascontiguousarray(pts, np.float32).tofile(f)
    from devil_ray_b200 import meshgen
    rgb = np.array(meshgen.TF_RGB, np.float32)
    alpha = np.array(meshgen.TF_ALPHA, np.float32)
    with open(d / "render.bin", "wb") as f:
        np.array([w, w, samples], np.int32).tofile(f)
        np.array([*CAM["pos"], *CAM["look_at"], *CAM["up"], CAM["fov"]], np.float32).tofile(f)
        np.asarray(light13, np.float32).reshape(13).tofile(f)
        np.array([rgb.shape[0]], np.int32).tofile(f)
        rgb.tofile(f)
        np.array([alpha.shape[0]], np.int32).tofile(f)
        alpha.tofile(f)
    return rgb, alpha


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["volume_8", "p3_6"])
def test_cpp_interface_matches_reference(cuda, ref, tmp_path, name):
    from devil_ray_b200 import meshgen
    from devil_ray_b200.render import Camera, PointLight
    if not EXE.exists():
        pytest.fail("C++ test program missing: build with make -C devil_ray_b200/cpp")
    m = meshgen.workload_mesh(name) if name != "p3_6" else \
        meshgen.warped_mesh(6, 3, 0.05, gaussian_field_seed=4)
    rng = np.random.default_rng(11)
    pts = rng.uniform(-0.05, 1.05, size=(20000, 3)).astype(np.float32)
    w, samples = 96, 300
    cam = Camera(w, w, CAM["pos"], CAM["look_at"], CAM["up"], CAM["fov"])
    light13 = PointLight.default(cam).as13()
    rgb, alpha = _write_inputs(tmp_path, m, pts, w, samples, light13)

    r = subprocess.run([str(EXE), str(tmp_path)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "ok" in r.stdout

    rm = ref.RefHexMesh(m.order, m.ctrl_idx, m.xyz, m.field)
    n = pts.shape[0]

    # Mesh::locate at the reference's own settings: same cells, ref points
    # within the Newton tolerance.
    raw = np.fromfile(tmp_path / "locate.bin", np.uint8)
    cell = raw[: 4 * n].view(np.int32)
    refp = raw[4 * n:].view(np.float32).reshape(n, 3)
    rcell, rref = rm.locate(pts)
    same = cell == rcell
    assert same.mean() > 0.999, f"{(~same).sum()} cell mismatches"
    both = same & (cell >= 0)
    assert np.abs(refp[both] - rref[both]).max() < 1e-3
    assert 0.3 < (cell >= 0).mean() < 1.0

    # PointLocation: field value at located points, empty value elsewhere.
    vals = np.fromfile(tmp_path / "pointloc.bin", np.float32)
    assert np.all(vals[cell < 0] == np.float32(-1e30))
    nd = (m.order + 1) ** 3
    conn = np.asarray(m.ctrl_idx, np.int64).reshape(-1, nd)
    fld = np.asarray(m.field, np.float32)
    for e in np.unique(cell[both])[:64]:
        sel = both & (cell == e)
        rv, _ = ref.eval_hex_scalar(m.order, fld[conn[e]], refp[sel])
        assert np.abs(vals[sel] - rv).max() < 1e-4

    # Volume::integrate + composite == reference volume image.
    img = np.fromfile(tmp_path / "volume.bin", np.float32).reshape(w, w, 4)
    rimg, _ = rm.volume(w, w, np.array([*CAM["pos"], *CAM["look_at"], *CAM["up"]], np.float32),
                        CAM["fov"], samples, True, 1024, rgb, alpha, light13[None])
    d = np.abs(img - rimg)
    bad = np.any(d > 1.0 / 255.0, axis=-1)
    print(f"volume: {bad.sum()} pixels > 1/255, max {d.max():.2e}")
    assert not bad.any(), f"volume: {bad.sum()} pixels > 1/255, max {d.max():.2e}"

    # MeshBoundary + Surface::nearest_hit/fragments/shade == reference.
    raw = np.fromfile(tmp_path / "surface.bin", np.float32)
    simg = raw[: 4 * w * w].reshape(w, w, 4)
    sdepth = raw[4 * w * w:].reshape(w, w)
    rs = rm.surface(w, w, np.array([*CAM["pos"], *CAM["look_at"], *CAM["up"]], np.float32),
                    CAM["fov"], 1024, rgb, alpha, light13[None])
    d = np.abs(simg - rs["rgba"])
    bad = np.any(d > 1.0 / 255.0, axis=-1)
    print(f"surface: {bad.sum()} pixels > 1/255, max {d.max():.2e}")
    assert not bad.any(), f"surface: {bad.sum()} pixels > 1/255, max {d.max():.2e}"
    hit = np.isfinite(rs["depth"]) & np.isfinite(sdepth) & (rs["depth"] < 1e30)
    assert np.abs(sdepth[hit] - rs["depth"][hit]).max() < 1e-3

    # ScalarRenderer: per-pixel depth, zone id and field value at the hit.
    raw = np.fromfile(tmp_path / "scalar.bin", np.uint8)
    npx = w * w
    sd = raw[: 4 * npx].view(np.float32)
    sz = raw[4 * npx: 8 * npx].view(np.int32)
    sv = raw[8 * npx:].view(np.float32)
    rd, rz, rv = rm.scalar_render(w, w, np.array([*CAM["pos"], *CAM["look_at"], *CAM["up"]],
                                                 np.float32), CAM["fov"])
    rd, rz, rv = rd.reshape(-1), rz.reshape(-1), rv.reshape(-1)
    same = sz == rz
    assert same.mean() > 0.995
    hitp = same & (sz >= 0)
    assert np.abs(sd[hitp] - rd[hitp]).max() < 1e-4
    assert np.abs(sv[hitp] - rv[hitp]).max() < 1e-4
    assert np.isnan(sd[sz < 0]).all() and np.isnan(sv[sz < 0]).all()

    # Lineout: points bit-identical, values equal (empty value outside).
    raw = np.fromfile(tmp_path / "lineout.bin", np.float32)
    lp = raw[: 3 * 4 * 39].reshape(-1, 3)
    lv = raw[3 * 4 * 39:]
    starts = [(0.0, 0.0, 0.0), (0.1, 0.5, 0.9), (-0.2, 0.3, 0.4), (0.5, 0.5, 1.3)]
    ends = [(1.0, 1.0, 1.0), (1.2, 0.5, 0.1), (1.1, 0.35, 0.45), (0.5, 0.5, -0.3)]
    rp, rv = rm.lineout(starts, ends, 37, -7.0)
    assert np.array_equal(lp.view(np.int32), rp.view(np.int32))
    out = rv == np.float32(-7.0)
    assert np.array_equal(lv == np.float32(-7.0), out)
    assert np.abs(lv[~out] - rv[~out]).max() < 1e-4


RENDER_EXE = ROOT / "devil_ray_b200" / "cpp" / "tests" / "t_dray_b200_render"


def _scene_domains(name):
    """(order, ctrl_idx, xyz, field) per domain: the mesh's elements split in
    two halves by element index for the two-domain scenes."""
    from devil_ray_b200 import meshgen
    if name == "two_domains":
        m = meshgen.warped_mesh(6, 2, 0.05, jitter=0.01, seed=2)
        nd = (m.order + 1) ** 3
        cut = (m.ctrl_idx.size // nd // 2) * nd
        return [(m.order, m.ctrl_idx[:cut], m.xyz, m.field),
                (m.order, m.ctrl_idx[cut:], m.xyz, m.field)]
    m = meshgen.warped_mesh(5, 3, 0.05, gaussian_field_seed=4)
    return [(m.order, m.ctrl_idx, m.xyz, m.field)]


def _write_scene(d, doms, w, cam9, fov, pads, elevate, azimuth, surface, surf_domains, draw_mesh,
                 thickness, volume, samples, lighting, tf_samples, rgb, alpha):
    with open(d / "scene.bin", "wb") as f:
        np.array([len(doms)], np.int32).tofile(f)
        for order, ci, xyz, fld in doms:
            nd = (order + 1) ** 3
            np.array([order, ci.size // nd, xyz.shape[0]], np.int32).tofile(f)
            np.ascontiguousarray(ci, np.int32).tofile(f)
            np.ascontiguousarray(xyz, np.float32).tofile(f)
            np.ascontiguousarray(fld, np.float32).tofile(f)
        np.array([w, w], np.int32).tofile(f)
        np.asarray(cam9, np.float32).tofile(f)
        np.array([fov], np.float32).tofile(f)
        np.array([pads is not None], np.int32).tofile(f)
        np.asarray(pads if pads is not None else (0, 0, 0), np.float64).tofile(f)
        np.array([elevate, azimuth], np.float32).tofile(f)
        np.array([surface, surf_domains[0], surf_domains[1], draw_mesh], np.int32).tofile(f)
        np.array([thickness], np.float32).tofile(f)
        np.array([volume, samples, lighting, tf_samples], np.int32).tofile(f)
        np.array([rgb.shape[0]], np.int32).tofile(f)
        rgb.tofile(f)
        np.array([alpha.shape[0]], np.int32).tofile(f)
        alpha.tofile(f)


SCENES = {
    # two domains, camera on the collection's padded bounds then turned; the
    # far domain's boundary surface and, composited in front of it, the
    # volume of both domains (a surface of the whole collection would hide
    # the volume behind its near faces)
    "two_domain_surface_volume": dict(mesh="two_domains", pads=(0.1, 0.05, 0.2), elevate=15.0,
                                      azimuth=30.0, surface=1, surf_domains=(0, 1), draw_mesh=0,
                                      volume=1, lighting=1),
    # two domains, both domains' boundary surfaces (their cut faces too)
    "two_domain_surfaces": dict(mesh="two_domains", pads=(0.0, 0.1, 0.0), elevate=-20.0,
                                azimuth=75.0, surface=1, surf_domains=(0, 2), draw_mesh=1,
                                volume=0, lighting=1),
    # one domain, mesh lines over the shaded boundary, the volume in front
    "mesh_lines": dict(mesh="one_domain", pads=None, elevate=0.0, azimuth=-20.0, surface=1,
                       surf_domains=(0, 1), draw_mesh=1, volume=1, lighting=1),
    # two domains, volume alone, unlit
    "two_domain_volume": dict(mesh="two_domains", pads=(0.0, 0.0, 0.0), elevate=-10.0,
                              azimuth=0.0, surface=0, surf_domains=(0, 0), draw_mesh=0, volume=1,
                              lighting=0),
}


@pytest.mark.gpu
@pytest.mark.parametrize("scene", list(SCENES))
def test_cpp_renderer_matches_reference(cuda, ref, tmp_path, scene):
    """Renderer::render through the C++ interface against the reference's own
    Renderer::render (colour bars off; its single-rank partial compositor is
    the Volume::save blend): camera moves bit for bit, framebuffer colours
    within 1/255 per channel, depths equal where both have a hit, and the
    PNG files Framebuffer::save / save_depth / Volume::save write decode to
    the framebuffers they were written from."""
    from devil_ray_b200 import meshgen
    from png_util import read_png_rgba, to_rgba8
    if not RENDER_EXE.exists():
        pytest.fail("C++ test program missing: build with make -C devil_ray_b200/cpp")
    sc = SCENES[scene]
    doms = _scene_domains(sc["mesh"])
    w, fov, samples, tf_samples, thickness = 128, 30.0, 300, 256, 0.08
    cam9 = np.array([*CAM["pos"], *CAM["look_at"], *CAM["up"]], np.float32)
    rgb = np.array(meshgen.TF_RGB, np.float32)
    alpha = np.array(meshgen.TF_ALPHA, np.float32)
    _write_scene(tmp_path, doms, w, cam9, fov, sc["pads"], sc["elevate"], sc["azimuth"],
                 sc["surface"], sc["surf_domains"], sc["draw_mesh"], thickness, sc["volume"],
                 samples, sc["lighting"], tf_samples, rgb, alpha)
    out = subprocess.run([str(RENDER_EXE), str(tmp_path)], capture_output=True, text=True,
                         timeout=300)
    assert out.returncode == 0, out.stderr
    raw = np.fromfile(tmp_path / "render.bin", np.float32)
    img = raw[:4 * w * w].reshape(w, w, 4)
    dep = raw[4 * w * w:].reshape(w, w)
    camf = np.fromfile(tmp_path / "camera.bin", np.float32)

    # the reference: its camera moves, its Renderer, its PNG writer
    bounds = None
    if sc["pads"] is not None:
        b6 = np.array([ref.RefHexMesh(o, ci, xyz).bvh()["bounds"] for o, ci, xyz, _ in doms])
        bounds = np.array([b6[:, 0].min(), b6[:, 1].max(), b6[:, 2].min(), b6[:, 3].max(),
                           b6[:, 4].min(), b6[:, 5].max()], np.float32)
    want_cam, want_fov = ref.camera_move(w, w, cam9, fov, bounds,
                                         sc["pads"] if sc["pads"] is not None else (0, 0, 0),
                                         sc["elevate"], sc["azimuth"])
    assert np.array_equal(camf[:6].view(np.uint32), want_cam[:6].view(np.uint32))
    assert camf[6] == np.float32(want_fov)
    rimg, rdep = ref.render_scene(doms, w, w, cam9, fov, pads=sc["pads"], elevate=sc["elevate"],
                                  azimuth=sc["azimuth"], surface=bool(sc["surface"]),
                                  surface_domains=sc["surf_domains"],
                                  draw_mesh=bool(sc["draw_mesh"]), line_thickness=thickness,
                                  volume=bool(sc["volume"]), samples=samples,
                                  use_lighting=bool(sc["lighting"]), tf_samples=tf_samples,
                                  rgb_pts=rgb, alpha_pts=alpha,
                                  save_prefix=tmp_path / "ref_render")
    d = np.abs(img - rimg)
    bad = np.any(d > 1.0 / 255.0, axis=-1)
    hit, rhit = np.isfinite(dep) & (dep < 1e30), np.isfinite(rdep) & (rdep < 1e30)
    print(f"{scene}: alpha>0 pixels {np.mean(img[..., 3] > 0):.3f}, "
          f"pixels > 1/255: {bad.sum()} of {bad.size}, max diff {d.max():.2e}, "
          f"depth coverage {hit.mean():.3f} vs {rhit.mean():.3f}")
    assert np.mean(img[..., 3] > 0) > 0.1
    assert not bad.any()
    both = hit & rhit
    assert not (hit != rhit).any()
    assert np.allclose(dep[both], rdep[both], rtol=1e-4, atol=1e-4)
    # the PNG files decode to what was rendered
    assert np.array_equal(read_png_rgba(tmp_path / "render.png"), to_rgba8(img))
    ref_png = read_png_rgba(tmp_path / "ref_render.png")
    assert np.array_equal(ref_png, to_rgba8(rimg))
    dpng = read_png_rgba(tmp_path / "render_depth.png")
    assert np.all(dpng[..., 3] == 255) and np.all(dpng[..., 0] == dpng[..., 1])
    if sc["mesh"] == "one_domain":
        # Volume::save of the single domain's partials against the
        # reference's Volume::integrate + save compositing on the same camera
        vimg = read_png_rgba(tmp_path / "volume.png")
        o, ci, xyz, fld = doms[0]
        from devil_ray_b200.render import Camera, PointLight
        cam = Camera(w, w, tuple(camf[:3]), tuple(camf[3:6]), CAM["up"], float(camf[6]))
        light = PointLight.default(cam)
        cam9m = np.array([*camf[:6], *CAM["up"]], np.float32)
        rv, _ = ref.RefHexMesh(o, ci, xyz, fld).volume(
            w, w, cam9m, float(camf[6]), samples, bool(sc["lighting"]), tf_samples, rgb, alpha,
            light.as13()[None])
        vd = np.abs(vimg.astype(np.int32) - to_rgba8(rv).astype(np.int32))
        print(f"{scene}: Volume::save pixels off by more than 1 level: "
              f"{np.any(vd > 1, axis=-1).sum()}")
        assert not np.any(vd > 1)
