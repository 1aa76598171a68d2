"""Queries on the GPU against the reference (oracle/_ref): Lineout sample
points bit-identical to Lineout::create_points, and the values along the
lines equal to Lineout::execute's (same empty value outside the mesh)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

LINES_START = [(0.0, 0.0, 0.0), (0.1, 0.5, 0.9), (-0.2, 0.3, 0.4), (0.5, 0.5, 1.3)]
LINES_END = [(1.0, 1.0, 1.0), (1.2, 0.5, 0.1), (1.1, 0.35, 0.45), (0.5, 0.5, -0.3)]


@pytest.mark.parametrize("name", ["volume_8", "p3_6"])
def test_lineout_matches_reference(cuda, ref, name):
    import torch
    from devil_ray_b200 import api, meshgen
    from devil_ray_b200.render import Lineout, UnstructuredField
    m = meshgen.workload_mesh(name) if name != "p3_6" else \
        meshgen.warped_mesh(6, 3, 0.05, gaussian_field_seed=4)
    r = ref.RefHexMesh(m.order, m.ctrl_idx, m.xyz, m.field)
    rp, rv = r.lineout(LINES_START, LINES_END, 37, -7.0)
    g = api.UnstructuredMesh(m.ctrl_idx, m.xyz, m.order, device=cuda)
    f = UnstructuredField(m.ctrl_idx, m.field, m.order, name="f", device=cuda)
    lo = Lineout()
    lo.samples(37)
    lo.empty_val(-7.0)
    for a, b in zip(LINES_START, LINES_END):
        lo.add_line(a, b)
    lo.add_var("f")
    lo.add_var("missing")
    pts, vals = lo.execute(g, {"f": f})
    torch.cuda.synchronize()
    p = pts.cpu().numpy()
    v = vals["f"].cpu().numpy()
    assert p.shape == rp.shape == (4 * 39, 3)
    assert np.array_equal(p.view(np.int32), rp.view(np.int32))
    outside = rv == np.float32(-7.0)
    assert np.array_equal(v == np.float32(-7.0), outside)
    assert np.abs(v[~outside] - rv[~outside]).max() < 1e-4
    print(f"{name}: {(~outside).sum()} of {len(v)} points inside, "
          f"max |v - v_ref| {np.abs(v[~outside] - rv[~outside]).max():.2e}")


def test_lineout_rejects_bad_input(cuda):
    from devil_ray_b200.render import Lineout
    lo = Lineout()
    with pytest.raises(ValueError):
        lo.samples(0)


@pytest.mark.parametrize("name", ["p3_8", "p2_8"])
def test_scalar_renderer_matches_reference(cuda, ref, name):
    """ScalarRenderer's per-pixel depth, zone id and field value equal the
    reference's nearest hits and fragments (rays on shared edges aside)."""
    import torch
    from devil_ray_b200 import api, meshgen
    from devil_ray_b200.render import (Camera, MeshBoundary, ScalarRenderer, Surface,
                                       UnstructuredField)
    m = meshgen.warped_mesh(8, 3, 0.08, jitter=0.01, seed=1) if name == "p3_8" else \
        meshgen.workload_mesh("volume_8")
    w = 128
    c = meshgen.CAMERA
    cam9 = np.array([*c["pos"], *c["look_at"], *c["up"]], np.float32)
    rd, rz, rs = ref.RefHexMesh(m.order, m.ctrl_idx, m.xyz, m.field).scalar_render(
        w, w, cam9, c["fov"])
    g = api.UnstructuredMesh(m.ctrl_idx, m.xyz, m.order, device=cuda)
    f = UnstructuredField(m.ctrl_idx, m.field, m.order, device=cuda)
    faces, ff = MeshBoundary().execute(g, f)
    sr = ScalarRenderer(Surface(faces, ff), {"f": ff})
    sr.field_names(["f", "missing"])
    buf = sr.render(Camera(w, w, c["pos"], c["look_at"], c["up"], c["fov"]))
    torch.cuda.synchronize()
    z = buf.zone_ids.cpu().numpy().reshape(w, w)
    d = buf.depths.cpu().numpy().reshape(w, w)
    s = buf.scalars["f"].cpu().numpy().reshape(w, w)
    assert "missing" not in buf.scalars
    same = z == rz
    assert same.mean() > 0.995, f"{(~same).sum()} zone mismatches"
    assert (np.isnan(d) != (rz < 0)).sum() <= 0.005 * d.size
    assert np.array_equal(np.isnan(d), z < 0) and np.array_equal(np.isnan(s), z < 0)
    hit = same & (z >= 0)
    assert np.abs(d[hit] - rd[hit]).max() < 1e-4
    assert np.abs(s[hit] - rs[hit]).max() < 1e-4
    print(f"{name}: hit pixels {(z >= 0).sum()}, zone mismatches {(~same).sum()}")
