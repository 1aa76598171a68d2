"""CPU tests of the oracle itself (no GPU): the reference build and the
restatement are pinned against the known answers of the reference's own
t_dray_external_evals fixture and against each other."""
import numpy as np
import pytest


def iota_known_answer(p, refs):
    """Control values 100, 101, ... (u fastest; the fixture of
    tests/dray/t_dray_external_evals.cpp) form an affine function of the
    control index, which Bernstein bases reproduce exactly:
    f = 100 + p u + p(p+1) v + p(p+1)^2 w, gradient (p, p(p+1), p(p+1)^2)."""
    u, v, w = refs[:, 0], refs[:, 1], refs[:, 2]
    f = 100 + p * u + p * (p + 1) * v + p * (p + 1) ** 2 * w
    g = np.array([p, p * (p + 1), p * (p + 1) ** 2], np.float64)
    return f, np.broadcast_to(g, refs.shape)


def sample_grid(p):
    t = np.arange(p + 1) / p
    w, v, u = np.meshgrid(t, t, t, indexing="ij")
    return np.stack([u.ravel(), v.ravel(), w.ravel()], 1)


@pytest.mark.parametrize("p", [1, 2, 3, 4, 5])
def test_reference_eval_known_answers(ref, p):
    vals = 100 + np.arange((p + 1) ** 3, dtype=np.float32)
    refs = sample_grid(p)
    f, g = iota_known_answer(p, refs)
    v, d = ref.eval_hex_scalar(p, vals, refs)
    # tolerances of the reference test (1e-4 values, 5e-4 derivatives) plus
    # a few FP32 ulps of the value for the higher orders (|f| up to 315)
    assert np.allclose(v, f, rtol=1e-6, atol=1e-4)
    assert np.allclose(d, g, rtol=2e-6, atol=5e-4)
    if p <= 2:
        vf, df = ref.eval_hex_scalar(p, vals, refs, fixed=True)
        assert np.allclose(vf, v, rtol=0, atol=4 * np.spacing(np.float32(f.max())))
        assert np.allclose(df, d, rtol=0, atol=1e-4)


@pytest.mark.parametrize("p", [1, 2, 3, 4, 5])
def test_restated_eval_known_answers(p):
    from oracle import restate
    if not restate.available():
        pytest.skip("restated oracle not built")
    vals = 100 + np.arange((p + 1) ** 3, dtype=np.float64)
    rng = np.random.default_rng(p)
    refs = np.concatenate([sample_grid(p), rng.uniform(0, 1, size=(50, 3))])
    f, g = iota_known_answer(p, refs)
    X, J = restate.hex_eval_d(p, vals, refs)
    assert np.abs(X[:, 0] - f).max() < 1e-9
    assert np.abs(J[:, :, 0] - g).max() < 1e-9


def test_restated_eval_matches_reference_random(ref):
    from oracle import restate
    rng = np.random.default_rng(3)
    for p in (1, 2, 3):
        vals = rng.uniform(-1, 1, size=(p + 1) ** 3).astype(np.float32)
        refs = rng.uniform(0, 1, size=(200, 3))
        v, d = ref.eval_hex_scalar(p, vals, refs.astype(np.float32))
        X, J = restate.hex_eval_d(p, vals.astype(np.float64), refs.astype(np.float32).astype(np.float64))
        assert np.abs(v - X[:, 0]).max() < 1e-5
        assert np.abs(d - J[:, :, 0]).max() < 5e-5


def test_restated_locate_matches_reference(ref):
    from devil_ray_b200 import meshgen
    from oracle import restate
    m = meshgen.workload_mesh("volume_8")
    r = ref.RefHexMesh(m.order, m.ctrl_idx, m.xyz, m.field)
    b = r.bvh()
    q = meshgen.uniform_queries(20000, 7)
    rc, rr = r.locate(q)
    oc, orf, it, ca = restate.locate(m.order, m.ctrl_idx, m.xyz, b, q, 1e-4, 20, 0)
    assert (rc == oc).mean() > 0.999
    hit = (rc == oc) & (rc >= 0)
    assert np.abs(rr[hit] - orf[hit]).max() < 1e-5
    assert 0.90 < (rc >= 0).mean() < 0.94  # ~8% of queries lie outside


def test_trilinear_mesh_has_positive_jacobian():
    from devil_ray_b200 import meshgen
    from oracle import restate
    for dist, seed in ((0.15, 2), (0.25, 3)):
        m = meshgen.trilinear_distorted_mesh(6, 2, dist, seed=seed)
        t = np.linspace(0, 1, 5)
        w, v, u = np.meshgrid(t, t, t, indexing="ij")
        refs = np.stack([u.ravel(), v.ravel(), w.ravel()], 1)
        nd = 27
        for e in range(m.n_elem):
            cp = m.xyz[m.ctrl_idx[e * nd:(e + 1) * nd]].astype(np.float64)
            _, J = restate.hex_eval_d(2, cp, refs)
            det = np.linalg.det(np.transpose(J, (0, 2, 1)))
            assert det.min() > 0, (dist, e)


def test_meshgen_shapes_and_outside_fraction():
    from devil_ray_b200 import meshgen
    m = meshgen.workload_mesh("volume_8")
    assert m.n_elem == 512 and m.n_ctrl == 17 ** 3 and m.ctrl_idx.size == 512 * 27
    assert m.xyz.min() == 0.0 and m.xyz.max() == 1.0
    q = meshgen.uniform_queries(200000, 1)
    outside = np.any((q < 0) | (q > 1), axis=1).mean()
    assert abs(outside - 0.08) < 0.005


def test_local_frame_newton_reaches_tolerance_on_fine_mesh(ref):
    """FP32 Newton in absolute coordinates stalls near tol 1e-5 once elements
    are small (rounding of X(r) ~ 1e-7 absolute, times 1/h in reference
    space); evaluated relative to each element's first control point, as the
    packed rows of the CUDA path are, it converges for every interior point."""
    from devil_ray_b200 import meshgen
    from oracle import restate
    if not restate.available():
        pytest.skip("restated oracle not built")
    m = meshgen.warped_mesh(40, 3, 0.05, gaussian_field_seed=4)
    b = ref.RefHexMesh(m.order, m.ctrl_idx, m.xyz, m.field).bvh()
    q = np.random.default_rng(3).uniform(0.001, 0.999, size=(40000, 3)).astype(np.float32)
    ca, ra, ia, _ = restate.locate(m.order, m.ctrl_idx, m.xyz, b, q, 1e-5, 20, 1)
    cl, rl, il, _ = restate.locate(m.order, m.ctrl_idx, m.xyz, b, q, 1e-5, 20, 1,
                                   local_frame=True)
    assert (cl >= 0).all()
    assert (ca < 0).sum() > 0          # the absolute form misses some
    assert il.mean() < ia.mean()
    both = (ca >= 0) & (ca == cl)
    assert np.abs(ra[both] - rl[both]).max() < 1e-4
    f64, ok = restate.newton_fp64(m.order, m.ctrl_idx, m.xyz, cl, q)
    assert np.abs(f64[ok] - rl[ok]).max() < 1e-5
