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
