"""LBVH parity on the GPU against the reference's own construct_bvh +
LinearBVHBuilder::construct (data_model/mesh_utils.cpp:514-677,
linear_bvh_builder.cpp:399-518), built from its sources in oracle/_ref.

Bar: sub-box AABBs, reference sub-boxes, scene bounds, Morton codes, the
sorted code sequence and the tree topology are bit-exact.  The reference
sorts with an unstable std::sort, so the leaf order inside runs of equal
codes may differ; those runs are compared as sets and counted, and inner
boxes are compared exactly for every node whose leaf range does not cut a
tie run.
"""
import numpy as np
import pytest

from tests.bvh_util import (node_children, node_leaf_ranges, subbox_aabbs, tie_runs)

pytestmark = pytest.mark.gpu

CASES = [("volume_8", None), ("trilinear_12", None), ("surface_32_small", None)]


def _mesh(name):
    from devil_ray_b200 import meshgen
    if name == "volume_8":
        return meshgen.workload_mesh("volume_8")
    if name == "trilinear_12":
        return meshgen.trilinear_distorted_mesh(12, 2, 0.15, seed=11)
    if name == "surface_32_small":
        return meshgen.warped_mesh(10, 3, 0.08, jitter=0.01, seed=5)
    if name == "order1":
        return meshgen.warped_mesh(9, 1, 0.05)
    raise KeyError(name)


@pytest.fixture(scope="module", params=["volume_8", "trilinear_12", "surface_32_small", "order1"])
def built(request, cuda, ref):
    import torch
    from devil_ray_b200 import api
    m = _mesh(request.param)
    r = ref.RefHexMesh(m.order, m.ctrl_idx, m.xyz, m.field)
    rb = r.bvh()
    g = api.UnstructuredMesh(m.ctrl_idx, m.xyz, m.order, device=cuda)
    b = g.build_bvh(keep_codes=True)
    b.widen()
    sub = api.elem_subboxes(g)
    torch.cuda.synchronize()
    gb = {"inner": b.inner_nodes.cpu().numpy(), "leaf_nodes": b.leaf_nodes.cpu().numpy(),
          "aabb_ids": b.aabb_ids.cpu().numpy(), "bounds": b.bounds,
          "ref_boxes": b.ref_boxes.cpu().numpy(),
          "codes": b.sorted_codes.cpu().numpy().view(np.uint32),
          "sub_aabbs": sub[0].cpu().numpy(), "sub_prim": sub[1].cpu().numpy(),
          "sub_bounds": sub[3].cpu().numpy(), "wide": b.wide_nodes.cpu().numpy(),
          "n_wide": b.n_wide, "wide_depth": b.wide_depth}
    return request.param, m, r, rb, gb


def test_subboxes_bit_exact(built):
    name, m, r, rb, gb = built
    ref_sub = subbox_aabbs(rb["inner"], rb["aabb_ids"])
    assert ref_sub.shape == gb["sub_aabbs"].shape
    assert np.array_equal(ref_sub.view(np.uint32), gb["sub_aabbs"].view(np.uint32)), \
        f"{name}: {np.sum(np.any(ref_sub != gb['sub_aabbs'], axis=1))} sub-boxes differ"
    assert np.array_equal(rb["ref_boxes"].view(np.uint32), gb["ref_boxes"].view(np.uint32))
    nb = 33
    assert np.array_equal(gb["sub_prim"], np.repeat(np.arange(m.n_elem, dtype=np.int32), nb))
    assert np.array_equal(rb["bounds"].view(np.uint32), gb["bounds"].view(np.uint32))
    assert np.array_equal(rb["bounds"].view(np.uint32), gb["sub_bounds"].view(np.uint32))


def test_morton_codes_bit_exact(built, ref):
    name, m, r, rb, gb = built
    ref_codes, ref_bounds = ref.morton(gb["sub_aabbs"])
    import torch
    from devil_ray_b200 import api
    a = torch.as_tensor(gb["sub_aabbs"]).cuda()
    bnd = torch.as_tensor(gb["sub_bounds"]).cuda()
    codes = api.morton_codes(a, bnd).cpu().numpy().view(np.uint32)
    assert np.array_equal(codes, ref_codes)
    assert np.array_equal(np.sort(ref_codes), gb["codes"])


def test_topology_bit_exact(built, ref):
    name, m, r, rb, gb = built
    rl, rr = node_children(rb["inner"])
    gl, gr = node_children(gb["inner"])
    assert np.array_equal(rl, gl) and np.array_equal(rr, gr), f"{name}: topology differs"


def test_leaves_and_inner_boxes(built, ref):
    name, m, r, rb, gb = built
    codes = gb["codes"]
    runs = tie_runs(codes)
    # outside tie runs the leaf order is unique
    in_run = np.zeros(codes.size, bool)
    for s, e in runs:
        in_run[s:e] = True
    assert np.array_equal(rb["aabb_ids"][~in_run], gb["aabb_ids"][~in_run])
    assert np.array_equal(rb["leaf_nodes"][~in_run], gb["leaf_nodes"][~in_run])
    for s, e in runs:
        assert sorted(rb["aabb_ids"][s:e]) == sorted(gb["aabb_ids"][s:e])
    lo, hi = node_leaf_ranges(gb["inner"])
    gl, gr = node_children(gb["inner"])
    ambiguous = np.zeros(gb["inner"].shape[0], bool)
    for kids in (gl, gr):
        leaf = kids < 0
        clo = np.where(leaf, -kids - 1, lo[np.maximum(kids, 0) // 4])
        chi = np.where(leaf, -kids - 1, hi[np.maximum(kids, 0) // 4])
        for s, e in runs:
            ambiguous |= ((clo > s) & (clo < e)) | ((chi >= s) & (chi < e - 1))
    same = np.all(rb["inner"][:, :12].view(np.uint32) == gb["inner"][:, :12].view(np.uint32), axis=1)
    assert np.all(same[~ambiguous]), f"{name}: {np.sum(~same[~ambiguous])} inner nodes differ"
    print(f"{name}: leaves {codes.size}, tie runs {len(runs)}, leaves in runs {int(in_run.sum())}, "
          f"nodes cutting a run {int(ambiguous.sum())}")


def test_bvh_deterministic(cuda):
    import torch
    from devil_ray_b200 import api
    m = _mesh("trilinear_12")
    g = api.UnstructuredMesh(m.ctrl_idx, m.xyz, m.order, device=cuda)
    a = g.build_bvh()
    b = g.build_bvh()
    torch.cuda.synchronize()
    # compare bits: leaf child ids stored as float bits are NaN patterns
    assert torch.equal(a.inner_nodes.view(torch.int32), b.inner_nodes.view(torch.int32))
    assert torch.equal(a.aabb_ids, b.aabb_ids)
    assert torch.equal(a.leaf_nodes, b.leaf_nodes)


def test_radix_sort_stable_and_sorted(cuda):
    import torch
    from devil_ray_b200 import api
    rng = np.random.default_rng(0)
    for n in [1, 7, 2048, 2049, 100000, 1 << 20]:
        keys = rng.integers(0, 1 << 12, size=n, dtype=np.int64).astype(np.uint32)
        vals = np.arange(n, dtype=np.int32)
        k, v = api.radix_sort_pairs(torch.as_tensor(keys.view(np.int32)).cuda(),
                                    torch.as_tensor(vals).cuda(), bits=12)
        k = k.cpu().numpy().view(np.uint32)
        v = v.cpu().numpy()
        order = np.argsort(keys, kind="stable")
        assert np.array_equal(k, keys[order])
        assert np.array_equal(v, order.astype(np.int32))


def test_empty_mesh_special_case(cuda):
    from devil_ray_b200 import api
    g = api.UnstructuredMesh(np.zeros(0, np.int32), np.zeros((0, 3), np.float32), 2, device=cuda)
    b = g.build_bvh()
    assert b.n_leaf == 2 and b.n_inner == 1
    l, r = node_children(b.inner_nodes.cpu().numpy())
    assert l[0] == -1 and r[0] == -2
    assert np.all(np.isinf(b.bounds))


def test_wide_tree_is_the_exact_collapse(built):
    """The 4-wide traversal tree equals the collapse of the binary tree:
    grandchild boxes copied bit for bit, left-to-right child codes, empty
    slots as inverted boxes."""
    from tests.bvh_util import widen
    name, m, r, rb, gb = built
    boxes, codes = widen(gb["inner"])
    assert gb["n_wide"] == boxes.shape[0]
    w = gb["wide"][: gb["n_wide"]]
    lo = w[:, 0:12].reshape(-1, 3, 4)   # [node, axis, child]
    hi = w[:, 12:24].reshape(-1, 3, 4)
    for a in range(3):
        assert np.array_equal(lo[:, a, :].view(np.int32), boxes[:, :, 2 * a].view(np.int32)), name
        assert np.array_equal(hi[:, a, :].view(np.int32), boxes[:, :, 2 * a + 1].view(np.int32)), name
    assert np.array_equal(w[:, 24:28].view(np.int32), codes)
    assert np.array_equal(w[:, 28].view(np.int32), (codes != np.iinfo(np.int32).min).sum(1))
    print(f"{name}: {gb['n_wide']} wide nodes for {gb['inner'].shape[0]} binary, "
          f"wide depth {gb['wide_depth']}")
