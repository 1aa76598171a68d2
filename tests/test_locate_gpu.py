"""Point-location parity on the GPU (drb_locate through the C-ABI) against
the reference's Mesh::locate (oracle/_ref) and the restated oracle.

Bar: located element ids identical except for points
on shared faces/edges (counted and checked to be within the is_inside band
of both elements); reference coordinates within 1e-5; the FP64 Newton error
of every GPU result is stated and bounded.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _setup(cuda, name, npts, seed):
    from devil_ray_b200 import api, meshgen
    if name == "volume_8":
        m = meshgen.workload_mesh("volume_8")
    elif name == "trilinear_12":
        m = meshgen.trilinear_distorted_mesh(12, 2, 0.15, seed=11)
    elif name == "trilinear_12_d25":
        m = meshgen.trilinear_distorted_mesh(12, 2, 0.25, seed=12)
    elif name == "p3_10":
        m = meshgen.warped_mesh(10, 3, 0.08, jitter=0.01, seed=5)
    elif name == "p1_9":
        m = meshgen.warped_mesh(9, 1, 0.05)
    q = meshgen.uniform_queries(npts, seed)
    g = api.UnstructuredMesh(m.ctrl_idx, m.xyz, m.order, device=cuda)
    return m, q, g


def _shared_face_ok(m, cell_a, ref_a, cell_b, ref_b, band=2e-3):
    """Both answers lie on the boundary band of their elements (a point on a
    face or edge shared by the two elements)."""
    def on_boundary(r):
        return np.any((r < band) | (r > 1.0 - band), axis=-1)
    ok = np.ones(cell_a.shape, bool)
    both = (cell_a >= 0) & (cell_b >= 0)
    ok[both] = on_boundary(ref_a[both]) & on_boundary(ref_b[both])
    one = (cell_a >= 0) ^ (cell_b >= 0)
    ra = np.where((cell_a >= 0)[:, None], ref_a, ref_b)
    ok[one] = on_boundary(ra[one])
    return ok


@pytest.mark.parametrize("name", ["volume_8", "trilinear_12", "trilinear_12_d25", "p3_10", "p1_9"])
def test_locate_matches_reference(cuda, ref, name):
    import torch
    from devil_ray_b200 import _lib as L
    m, q, g = _setup(cuda, name, 40000, 7)
    r = ref.RefHexMesh(m.order, m.ctrl_idx, m.xyz, m.field)
    rc, rr = r.locate(q)
    # reference settings: tol 1e-4, 20 steps, zero-initialised guess
    cell, rf = g.locate(q, tol=1e-4, max_steps=20, guess_mode=L.GUESS_ZERO)
    torch.cuda.synchronize()
    cell = cell.cpu().numpy()
    rf = rf.cpu().numpy()
    same = cell == rc
    diff = ~same
    assert _shared_face_ok(m, cell[diff], rf[diff], rc[diff], rr[diff]).all(), \
        f"{name}: {diff.sum()} mismatches not on shared faces"
    assert diff.mean() < 2e-3, f"{name}: {diff.sum()} cell mismatches"
    hit = same & (cell >= 0)
    err = np.abs(rf[hit] - rr[hit]).max()
    assert err < 1e-5, f"{name}: max ref diff {err}"
    print(f"{name}: located {np.mean(cell >= 0):.4f}, cell mismatches {diff.sum()} "
          f"(shared faces), max |ref - ref_ref| {err:.2e}")


@pytest.mark.parametrize("name", ["volume_8", "trilinear_12_d25"])
@pytest.mark.parametrize("guess", ["center", "subref"])
def test_locate_tol_1e5_vs_restated_and_fp64(cuda, name, guess):
    import torch
    from devil_ray_b200 import _lib as L
    from oracle import restate
    if not restate.available():
        pytest.skip("restated oracle not built")
    m, q, g = _setup(cuda, name, 30000, 9)
    mode = L.GUESS_ELEM_CENTER if guess == "center" else L.GUESS_SUBREF_CENTER
    cell, rf, it, ca, nd = g.locate(q, tol=1e-5, max_steps=20, guess_mode=mode, stats=True)
    torch.cuda.synchronize()
    b = g.get_bvh()
    bvh = {"inner": b.inner_nodes.cpu().numpy(), "leaf_nodes": b.leaf_nodes.cpu().numpy(),
           "aabb_ids": b.aabb_ids.cpu().numpy(), "ref_boxes": b.ref_boxes.cpu().numpy()}
    # the packed rows evaluate in each element's local frame; so does the oracle here
    oc, orf, oit, oca = restate.locate(m.order, m.ctrl_idx, m.xyz, bvh, q, 1e-5, 20, mode,
                                       local_frame=True)
    cell = cell.cpu().numpy()
    rf = rf.cpu().numpy()
    same = cell == oc
    assert (~same).mean() < 2e-3
    assert _shared_face_ok(m, cell[~same], rf[~same], oc[~same], orf[~same]).all()
    hit = same & (cell >= 0)
    assert np.abs(rf[hit] - orf[hit]).max() < 1e-5
    # same traversal -> same candidate counts except where the result differs
    assert np.array_equal(ca.cpu().numpy()[same], oca[same])
    # FP64 error of the GPU solution
    f64, ok = restate.newton_fp64(m.order, m.ctrl_idx, m.xyz, cell, q)
    e = np.abs(f64[(cell >= 0) & ok] - rf[(cell >= 0) & ok]).max()
    assert e < 1e-5, f"FP64 error {e}"
    print(f"{name}/{guess}: mean iters {it.float().mean().item():.3f}, FP64 max err {e:.2e}")


def test_locate_edge_cases(cuda):
    import torch
    from devil_ray_b200 import _lib as L
    m, q, g = _setup(cuda, "volume_8", 10, 1)
    # empty query
    c, r = g.locate(np.zeros((0, 3), np.float32))
    assert c.numel() == 0
    # far outside, NaN and the exact corners / centre
    pts = np.array([[5, 5, 5], [-1, 0.5, 0.5], [np.nan, 0.5, 0.5], [0, 0, 0], [1, 1, 1],
                    [0.5, 0.5, 0.5]], np.float32)
    c, r = g.locate(pts, guess_mode=L.GUESS_ZERO)
    c = c.cpu().numpy()
    assert c[0] == -1 and c[1] == -1 and c[2] == -1
    assert c[3] >= 0 and c[4] >= 0 and c[5] >= 0
    with pytest.raises(L.DrbError):
        g.locate(pts, tol=-1.0)
    with pytest.raises(L.DrbError):
        g.locate(pts, guess_mode=L.GUESS_GIVEN)


def test_local_frame_locates_fine_order3_mesh(cuda):
    """On a 48^3 order-3 mesh the FP32 rounding of absolute coordinates puts
    Newton's step noise near the 1e-5 tolerance, and the reference-style
    solve misses interior points; the packed rows' local frame locates
    every one, each checked against the FP64 solution."""
    import torch
    from devil_ray_b200 import _lib as L
    from devil_ray_b200 import api, meshgen
    from oracle import restate
    if not restate.available():
        pytest.skip("restated oracle not built")
    m = meshgen.warped_mesh(48, 3, 0.05, gaussian_field_seed=4)
    g = api.UnstructuredMesh(m.ctrl_idx, m.xyz, m.order, device=cuda)
    q = np.random.default_rng(21).uniform(0.001, 0.999, size=(40000, 3)).astype(np.float32)
    cell, rf, it, ca, nd = g.locate(q, tol=1e-5, max_steps=20, guess_mode=L.GUESS_ELEM_CENTER,
                                    stats=True)
    torch.cuda.synchronize()
    cell = cell.cpu().numpy()
    rf = rf.cpu().numpy()
    assert (cell >= 0).all(), f"{(cell < 0).sum()} interior points not located"
    f64, ok = restate.newton_fp64(m.order, m.ctrl_idx, m.xyz, cell, q)
    assert ok.all()
    e = np.abs(f64 - rf).max()
    assert e < 1e-5, f"FP64 error {e}"
    b = g.get_bvh()
    bvh = {"inner": b.inner_nodes.cpu().numpy(), "leaf_nodes": b.leaf_nodes.cpu().numpy(),
           "aabb_ids": b.aabb_ids.cpu().numpy(), "ref_boxes": b.ref_boxes.cpu().numpy()}
    oc, orf, oit, oca = restate.locate(m.order, m.ctrl_idx, m.xyz, bvh, q, 1e-5, 20,
                                       L.GUESS_ELEM_CENTER, local_frame=True)
    same = cell == oc
    assert (~same).mean() < 2e-3
    assert _shared_face_ok(m, cell[~same], rf[~same], oc[~same], orf[~same]).all()
    ac, *_ = restate.locate(m.order, m.ctrl_idx, m.xyz, bvh, q, 1e-5, 20, L.GUESS_ELEM_CENTER)
    print(f"48^3 P3: mean iters {it.float().mean().item():.3f}, FP64 max err {e:.2e}; "
          f"absolute-coordinate FP32 Newton misses {(ac < 0).sum()} of {len(q)}")


@pytest.mark.parametrize("name", ["volume_8", "p3_10", "p1_9"])
def test_wide_traversal_equals_binary(cuda, name):
    """The batched kernel over the 4-wide tree returns exactly what it
    returns over the binary tree: cells, reference points (bit for bit),
    Newton iterations and candidate counts; only node visits differ."""
    import torch
    from devil_ray_b200 import api
    m, q, g = _setup(cuda, name, 50000, 13)
    b = g.get_bvh()
    assert b.wide_nodes is not None
    wide = api.BatchedLocator(g, tol=1e-5, max_steps=20, bvh=b)
    binary = api.BatchedLocator(g, tol=1e-5, max_steps=20, bvh=b.binary_only())
    c0, r0, i0, a0, n0 = binary.locate(q, stats=True)
    c1, r1, i1, a1, n1 = wide.locate(q, stats=True)
    torch.cuda.synchronize()
    assert torch.equal(c0, c1)
    assert torch.equal(r0.view(torch.int32), r1.view(torch.int32))
    assert torch.equal(i0, i1) and torch.equal(a0, a1)
    print(f"{name}: nodes visited binary {n0.float().mean().item():.2f}, "
          f"wide {n1.float().mean().item():.2f}")


def test_locate_host_equals_device_batched(cuda):
    """drb_locate_host (chunked, copies overlapped on three streams) gives
    the batched locate's results, for chunk sizes that do and do not divide
    the batch."""
    import torch
    from devil_ray_b200 import api
    m, q, g = _setup(cuda, "volume_8", 100000, 17)
    loc = api.BatchedLocator(g, tol=1e-5, max_steps=20)
    c0, r0 = loc.locate(q)
    torch.cuda.synchronize()
    hq = torch.from_numpy(np.ascontiguousarray(q, np.float32)).pin_memory()
    for chunk in (0, 30000, 1 << 20):
        hc = torch.empty(q.shape[0], dtype=torch.int32).pin_memory()
        hr = torch.empty((q.shape[0], 3), dtype=torch.float32).pin_memory()
        loc.locate_host(hq, out=(hc, hr), chunk=chunk)
        assert torch.equal(hc, c0.cpu())
        assert torch.equal(hr.view(torch.int32), r0.cpu().view(torch.int32))


@pytest.mark.parametrize("name", ["volume_8", "p3_10", "p1_9"])
def test_row_modes_identical(cuda, name):
    """The three places a candidate's control points can be read from during
    its Newton solve (L1 on every step, registers, warp-shared rows in shared
    memory) give bit-identical results and statistics."""
    import torch
    from devil_ray_b200 import _lib as L
    from devil_ray_b200 import api
    m, q, g = _setup(cuda, name, 50000, 19)
    out = []
    for mode in (0, 1, 2):
        for block in (64, 128):
            loc = api.BatchedLocator(g, tol=1e-5, max_steps=20,
                                     config=L.DrbLocateConfig(block, 0, 32, 1, mode))
            out.append(loc.locate(q, stats=True))
    torch.cuda.synchronize()
    c0, r0, i0, a0, n0 = out[0]
    for c, r, i, a, nd in out[1:]:
        assert torch.equal(c, c0)
        assert torch.equal(r.view(torch.int32), r0.view(torch.int32))
        assert torch.equal(i, i0) and torch.equal(a, a0) and torch.equal(nd, n0)


@pytest.mark.gpu
@pytest.mark.parametrize("shape", ["hex", "tet"])
def test_locate_graph_replay_matches_eager(cuda, shape):
    """The batched locate captured into a CUDA graph (BatchedLocator.capture)
    gives the eager results bit for bit on new queries at every replay."""
    import torch
    from devil_ray_b200 import _lib as L
    from devil_ray_b200 import api, meshgen
    if shape == "hex":
        m = meshgen.trilinear_distorted_mesh(12, 2, 0.15, seed=11)
        g = api.UnstructuredMesh(m.ctrl_idx, m.xyz, m.order, device=cuda)
    else:
        m = meshgen.tet_warped_mesh(6, 2, 0.05, jitter=0.01, seed=5)
        g = api.UnstructuredMesh(m.ctrl_idx, m.xyz, m.order, device=cuda, shape=L.SHAPE_SIMPLEX)
    loc = api.BatchedLocator(g, tol=1e-5, max_steps=20)
    n = 50000
    lg = loc.capture(n)
    for seed in (3, 4, 5):
        q = meshgen.uniform_queries(n, seed)
        c1, r1 = lg.run(q)
        c1, r1 = c1.clone(), r1.clone()
        c0, r0 = loc.locate(q)
        torch.cuda.synchronize()
        assert torch.equal(c0, c1)
        assert torch.equal(r0.view(torch.int32), r1.view(torch.int32))
        assert (c1 >= 0).float().mean() > 0.85


@pytest.mark.parametrize("name", ["volume_8", "p3_10", "p1_9"])
@pytest.mark.parametrize("guess", ["centre", "subref"])
def test_staged_equals_ordered_and_plain(cuda, name, guess):
    """Every placement of the queries and results (read through the Morton
    order, staged records, staged results) and the caller-ordered path
    (drb_locate_ordered) give the plain one-thread-per-query kernel's
    answers bit for bit, statistics included."""
    import torch
    from devil_ray_b200 import _lib as L
    from devil_ray_b200 import api
    m, q, g = _setup(cuda, name, 60000, 23)
    mode = L.GUESS_ELEM_CENTER if guess == "centre" else L.GUESS_SUBREF_CENTER
    loc = api.BatchedLocator(g, tol=1e-5, max_steps=20, guess_mode=mode)
    c0, r0, i0, a0, n0 = loc.locate(q, stats=True)
    order = loc.order(q)
    c1, r1, i1, a1, n1 = loc.locate(q, order=order, stats=True)
    c2, r2 = g.locate(q, tol=1e-5, max_steps=20, guess_mode=mode)
    # query records staged first (sort_queries 2), results staged as well
    # and put back by a separate pass (3)
    out = []
    for mode_s in (2, 3):
        loc_s = api.BatchedLocator(g, tol=1e-5, max_steps=20, guess_mode=mode,
                                   config=L.DrbLocateConfig(128, 0, 64, mode_s, 0))
        out.append(loc_s.locate(q, stats=True))
    torch.cuda.synchronize()
    for c, r in ((c1, r1), (c2, r2)) + tuple((o[0], o[1]) for o in out):
        assert torch.equal(c0, c)
        assert torch.equal(r0.view(torch.int32), r.view(torch.int32))
    for i, a, nd in ((i1, a1, n1),) + tuple((o[2], o[3], o[4]) for o in out):
        assert torch.equal(i0, i) and torch.equal(a0, a) and torch.equal(n0, nd)


@pytest.mark.parametrize("n", [1000, 80000, 2500000])
def test_stage_records_and_staged_kernel(cuda, n):
    """drb_query_stage lists every query once, cell by cell along the Morton
    curve, with its input index in w; drb_locate_staged on those records
    gives each query the answer drb_locate_batched gives it.  The sizes
    take the staging with no fine bits (one pass), one and three."""
    import torch
    from devil_ray_b200 import api
    m, q, g = _setup(cuda, "trilinear_12", n, 29)
    loc = api.BatchedLocator(g, tol=1e-5, max_steps=20)
    rec = loc.stage(q)
    res = loc.locate_staged(rec, records=True)
    cs, rs = loc.locate_staged(rec)
    c0, r0 = loc.locate(q)
    torch.cuda.synchronize()
    assert torch.equal(cs, c0) and torch.equal(rs.view(torch.int32), r0.view(torch.int32))
    idx = rec[:, 3].contiguous().view(torch.int32).long()
    assert torch.equal(torch.sort(idx).values, torch.arange(q.shape[0], device=cuda))
    qd = torch.as_tensor(q, device=cuda)
    assert torch.equal(rec[:, :3].contiguous().view(torch.int32), qd[idx].view(torch.int32))
    cell_of = res[:, 0].contiguous().view(torch.int32)
    assert torch.equal(cell_of, c0[idx])
    assert torch.equal(res[:, 1:].contiguous().view(torch.int32), r0[idx].view(torch.int32))
    code = _morton_cells(rec[:, :3].cpu().numpy(), g.get_bvh().bounds)
    assert np.all(np.diff(code) >= 0)


def _morton_cells(p, bounds):
    """Morton code (x lowest) of each point's query-order cell over the BVH
    bounds, 3..7 bits per axis so that a cell holds about eight queries."""
    n = p.shape[0]
    bits = 3
    while bits < 7 and (8 << (3 * bits)) < n:
        bits += 1
    code = np.zeros(n, np.int64)
    for k in range(3):
        lo, hi = np.float32(bounds[2 * k]), np.float32(bounds[2 * k + 1])
        sc = np.float32(1.0) / np.float32(hi - lo)
        t = ((p[:, k].astype(np.float32) - lo) * sc).astype(np.float32) * np.float32(1 << bits)
        t = np.minimum(np.maximum(t, np.float32(0)), np.float32((1 << bits) - 1))
        x = np.where(np.isnan(t), 0, t).astype(np.int64)
        for b in range(bits):
            code |= ((x >> b) & 1) << (3 * b + k)
    return code


def test_autotuner_config_is_valid_and_exact(cuda):
    """drb_locate_tune returns a launch shape from its candidate set, and the
    tuned locate's results equal the default shape's bit for bit."""
    import torch
    from devil_ray_b200 import api
    m, q, g = _setup(cuda, "trilinear_12", 120000, 31)
    base = api.BatchedLocator(g, tol=1e-5, max_steps=20)
    c0, r0 = base.locate(q)
    tuned = api.BatchedLocator(g, tol=1e-5, max_steps=20)
    cfg, ms = tuned.tune(q[:50000])
    assert cfg.block in (64, 128, 256) and cfg.blocks_per_sm in (0, 2, 4)
    assert cfg.chunk in (32, 64, 128, 256) and cfg.reg_elements in (0, 1, 2)
    assert cfg.sort_queries == 1 and ms > 0.0
    c1, r1 = tuned.locate(q)
    torch.cuda.synchronize()
    assert torch.equal(c0, c1)
    assert torch.equal(r0.view(torch.int32), r1.view(torch.int32))


@pytest.mark.parametrize("name", ["trilinear_12", "p3_10", "p1_9"])
def test_leaf_maps_match_fp64(cuda, name):
    """drb_bvh_leaf_maps on a hex mesh: each sampled leaf's record holds its
    sub-box centre, the element map there and the inverse Jacobian, against
    an FP64 evaluation of the same element at the same point."""
    import torch
    from tests.bvh_util import leaf_maps_fp64
    m, _, g = _setup(cuda, name, 16, 1)
    b = g.get_bvh()
    b.build_leaf_maps(g)
    torch.cuda.synchronize()
    maps = b.leaf_maps.cpu().numpy()
    leaves = np.random.default_rng(6).choice(b.n_leaf, 3000, replace=False)
    want = leaf_maps_fp64("hex", m.order, m.ctrl_idx, m.xyz, b, leaves)
    got = maps[leaves, :15]
    assert np.array_equal(got[:, :3], want[:, :3].astype(np.float32))
    assert np.abs(got[:, 3:6] - want[:, 3:6]).max() < 1e-5
    scale = np.abs(want[:, 6:]).max(axis=1, keepdims=True)
    assert (np.abs(got[:, 6:] - want[:, 6:]) / scale).max() < 1e-4


@pytest.mark.parametrize("name", ["trilinear_12", "trilinear_12_d25", "p3_10", "p1_9"])
def test_subbox_linear_guess(cuda, name):
    """The first guess from each leaf's linearised element map
    (GUESS_SUBBOX_LINEAR) converges to the same answers as the element-centre
    guess (same cells except on shared faces, reference points within the
    1e-5 tolerance, FP64 error below 1e-5), with fewer Newton steps than the
    sub-box-centre guess; the plain and batched kernels agree bit for bit."""
    import torch
    from devil_ray_b200 import _lib as L
    from devil_ray_b200 import api
    from oracle import restate
    m, q, g = _setup(cuda, name, 60000, 37)
    lin = api.BatchedLocator(g, tol=1e-5, max_steps=20, guess_mode=L.GUESS_SUBBOX_LINEAR)
    c4, r4, i4, a4, _ = lin.locate(q, stats=True)
    assert g.get_bvh().leaf_maps is not None
    cp, rp = g.locate(q, tol=1e-5, max_steps=20, guess_mode=L.GUESS_SUBBOX_LINEAR)
    c1, r1, i1, *_ = api.BatchedLocator(g, 1e-5, 20, L.GUESS_ELEM_CENTER).locate(q, stats=True)
    c2, r2, i2, *_ = api.BatchedLocator(g, 1e-5, 20, L.GUESS_SUBREF_CENTER).locate(q, stats=True)
    torch.cuda.synchronize()
    assert torch.equal(c4, cp) and torch.equal(r4.view(torch.int32), rp.view(torch.int32))
    c4n, r4n, c1n, r1n = c4.cpu().numpy(), r4.cpu().numpy(), c1.cpu().numpy(), r1.cpu().numpy()
    same = c4n == c1n
    assert (~same).mean() < 2e-3
    assert _shared_face_ok(m, c4n[~same], r4n[~same], c1n[~same], r1n[~same]).all()
    hit = same & (c4n >= 0)
    assert np.abs(r4n[hit] - r1n[hit]).max() < 1e-5
    if restate.available():
        f64, ok = restate.newton_fp64(m.order, m.ctrl_idx, m.xyz, c4n, q)
        sel = (c4n >= 0) & ok
        assert np.abs(f64[sel] - r4n[sel]).max() < 1e-5
    loc = c4 >= 0
    m4, m2, m1 = (float(i[loc].float().mean()) for i in (i4, i2, i1))
    print(f"{name}: mean Newton steps: sub-box linear {m4:.3f}, sub-box centre {m2:.3f}, "
          f"element centre {m1:.3f}")
    assert m4 < m2
