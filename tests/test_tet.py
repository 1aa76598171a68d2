"""Tet (simplex) elements on the CPU: the oracle pinned against the
reference built from its sources (oracle/_ref), and two defects of the
reference's simplex code that decide what the CUDA path restates.

  - construct_bvh sub-boxes of tets (mesh_utils.cpp:514-677 with
    pick_binary_split<Simplex> :455-480, split_subref<Simplex>
    ref_space.hpp:133-146, split_inplace<3,Simplex> elem_ops.hpp:1270-1311):
    the restatement with the reference's own dof indexing reproduces the
    reference's boxes bit for bit at orders 1 and 2 (order 3: all but the
    boxes touched by the reference's write past an element's scratch).
  - cartesian_to_tet_idx (elem_ops.hpp:32-47) is not the dof layout the
    evaluators walk for orders >= 2, so the CUDA path splits with the
    layered layout; at order 1 both give the same boxes.
  - Element<3,ncomp,Simplex,Linear>::eval_d (elem_ops.hpp:785-815) writes all
    three derivatives into out_deriv[0] and leaves C[3] out; the
    general-order evaluator is correct and is the one restated.
"""
import numpy as np
import pytest

from devil_ray_b200 import meshgen


def _tet_index_reference(i, j, k, p):
    e = p + 1
    return (((-1 - e) * 3 + k) * k + (3 * e + 6) * e + 2) * k // 6 + (2 * e + 1 - j) * j // 2 + i


def test_tet_generator_is_conforming_and_fills_the_cube():
    for p in (1, 2, 3):
        m = meshgen.tet_warped_mesh(3, p, 0.0)
        nd = meshgen.tet_dofs(p)
        conn = m.ctrl_idx.reshape(-1, nd)
        assert conn.shape[0] == 6 * 27
        # corner dofs of the layered layout: origin, u, v, w vertices
        corners = [0, p, (p + 1) * (p + 2) // 2 - 1, nd - 1]
        v = m.xyz[conn[:, corners]].astype(np.float64)            # [n, 4, 3]
        d = np.linalg.det(np.stack([v[:, 1] - v[:, 0], v[:, 2] - v[:, 0], v[:, 3] - v[:, 0]], -1))
        assert np.all(np.abs(d) > 0)
        assert abs(np.abs(d).sum() / 6.0 - 1.0) < 1e-6           # volumes sum to the cube
        # every interior triangle face is shared by exactly two tets
        faces = {}
        for e in range(conn.shape[0]):
            vv = conn[e, corners]
            for f in ((0, 1, 2), (0, 1, 3), (0, 2, 3), (1, 2, 3)):
                key = tuple(sorted(vv[list(f)]))
                faces[key] = faces.get(key, 0) + 1
        assert max(faces.values()) == 2
        n_boundary = sum(1 for c in faces.values() if c == 1)
        assert n_boundary == 6 * 2 * 9                           # 2 triangles per boundary square


def test_reference_tet_index_is_not_the_layered_layout():
    # the layered layout (dof order of the general-order evaluator)
    for p in (1, 2, 3):
        mi = meshgen.tet_multi_indices(p)
        assert len(mi) == meshgen.tet_dofs(p)
        ref = [_tet_index_reference(i, j, k, p) for (i, j, k) in mi]
        if p == 1:
            assert ref == list(range(len(mi)))
        else:
            assert ref != list(range(len(mi)))
    # order 2: (0,1,1) and (0,0,2) collide; order 3 reaches index 20 of 20 dofs
    assert _tet_index_reference(0, 1, 1, 2) == _tet_index_reference(0, 0, 2, 2) == 9
    assert max(_tet_index_reference(i, j, k, 3) for (i, j, k) in meshgen.tet_multi_indices(3)) == 20


@pytest.mark.parametrize("p", [1, 2])
def test_restated_tet_subboxes_match_reference(ref, p):
    """Orders 1-2 only: at order 3 the reference's split writes dof 20 of a
    20-dof box, past the end of its scratch array for the last box of the
    last element (a heap overflow that can crash the process), so the
    reference's order-3 tet BVH is not run."""
    from oracle import restate
    from tests.bvh_util import subbox_aabbs
    m = meshgen.tet_warped_mesh(3, p, 0.05, jitter=0.01, seed=3)
    r = ref.RefTetMesh(p, m.ctrl_idx, m.xyz, m.field)
    b = r.bvh()
    ref_aabbs = subbox_aabbs(b["inner"], b["aabb_ids"])
    a1, r1 = restate.tet_subboxes(p, m.ctrl_idx, m.xyz, reference_index=True)
    assert np.array_equal(b["ref_boxes"].view(np.int32), r1.view(np.int32))
    assert np.array_equal(ref_aabbs.view(np.int32), a1.view(np.int32))
    a0, r0 = restate.tet_subboxes(p, m.ctrl_idx, m.xyz, reference_index=False)
    if p == 1:
        assert np.array_equal(a0.view(np.int32), a1.view(np.int32))
        assert np.array_equal(r0.view(np.int32), r1.view(np.int32))
    else:
        assert not np.array_equal(a0.view(np.int32), a1.view(np.int32))


@pytest.mark.parametrize("p", [1, 2, 3])
def test_restated_tet_subboxes_bound_their_sub_simplices(p):
    from oracle import restate
    m = meshgen.tet_warped_mesh(3, p, 0.05, jitter=0.01, seed=3)
    a0, r0 = restate.tet_subboxes(p, m.ctrl_idx, m.xyz, reference_index=False)
    # with the layered layout every sub-box holds the geometry of its
    # sub-simplex: points sampled in each sub-simplex map into its box
    from oracle import restate as rs
    nd = meshgen.tet_dofs(p)
    conn = m.ctrl_idx.reshape(-1, nd)
    rng = np.random.default_rng(5)
    for e in range(0, conn.shape[0], 17):
        cp = m.xyz[conn[e]].astype(np.float64)
        for b_i in range(33):
            o = e * 33 + b_i
            verts = r0[o].reshape(4, 3).astype(np.float64)    # u, v, w vertices, origin
            lam = rng.dirichlet(np.ones(4), size=16)
            refp = lam @ verts
            X, _ = rs.tet_eval_d(p, cp, refp)
            lo, hi = a0[o, 0::2], a0[o, 1::2]
            assert np.all(X >= lo - 1e-6) and np.all(X <= hi + 1e-6)


@pytest.mark.parametrize("p", [1, 2, 3])
def test_restated_tet_eval_matches_reference_general_order(ref, p):
    from oracle import restate
    rng = np.random.default_rng(p)
    nd = meshgen.tet_dofs(p)
    vals = rng.normal(size=nd).astype(np.float32)
    lam = rng.dirichlet(np.ones(4), size=200)
    refp = lam[:, :3].astype(np.float32)
    rv, rd = ref.eval_tet_scalar(p, vals, refp, fixed=False)
    X, J = restate.tet_eval_d(p, vals.astype(np.float64), refp.astype(np.float64))
    assert np.abs(rv - X[:, 0]).max() < 1e-5
    assert np.abs(rd - J[:, :, 0]).max() < 1e-4
    if p == 2:
        # the fixed-order quadratic element agrees as well
        fv, fd = ref.eval_tet_scalar(p, vals, refp, fixed=True)
        assert np.abs(fv - X[:, 0]).max() < 1e-5
        assert np.abs(fd - J[:, :, 0]).max() < 1e-4


def test_reference_fixed_linear_tet_derivative_defect(ref):
    """The fixed-order Linear tet leaves d/dv and d/dw unset and drops C[3]
    from d/du; its value is right.  Its point location therefore fails, so
    order-1 tets are compared against the general-order element type."""
    from oracle import restate
    vals = np.array([1.0, 2.0, 5.0, 11.0], np.float32)
    refp = np.array([[0.2, 0.3, 0.1]], np.float32)
    fv, fd = ref.eval_tet_scalar(1, vals, refp, fixed=True)
    X, J = restate.tet_eval_d(1, vals.astype(np.float64), refp.astype(np.float64))
    assert abs(fv[0] - X[0, 0]) < 1e-6
    assert np.allclose(J[0, :, 0], [1.0, 4.0, 10.0])
    assert not np.allclose(fd[0], J[0, :, 0])
    m = meshgen.tet_warped_mesh(3, 1, 0.0)
    pts = np.random.default_rng(2).uniform(0.05, 0.95, size=(500, 3)).astype(np.float32)
    cell_fixed, _ = ref.RefTetMesh(1, m.ctrl_idx, m.xyz, fixed=True).locate(pts)
    cell_gen, _ = ref.RefTetMesh(1, m.ctrl_idx, m.xyz, fixed=False).locate(pts)
    assert (cell_gen >= 0).all()
    assert (cell_fixed < 0).mean() > 0.9
