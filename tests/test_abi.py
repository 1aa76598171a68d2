"""C-ABI boundary checks that need no GPU: the library loads, exports every
symbol declared in include/drb.h, and the pure host-side queries work."""
import ctypes as C

import numpy as np
import pytest


def test_library_exports_declared_symbols():
    from devil_ray_b200 import _lib as L
    lib = L.lib()
    names = L.declared_symbols()
    assert len(names) >= 8
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, f"libdrb.so lacks {missing}"


def test_host_queries():
    from devil_ray_b200 import _lib as L
    lib = L.lib()
    assert lib.drb_version() >= 1
    # geometry rows: 3 nd relative coordinates + the 3-float origin, padded to 4
    assert lib.drb_packed_stride(3, 2, 3) == 84
    assert lib.drb_packed_stride(3, 3, 3) == 196
    assert lib.drb_packed_stride(3, 1, 3) == 28
    assert lib.drb_packed_stride(3, 1, 1) == 8
    assert lib.drb_packed_stride(2, 3, 3) == 52
    assert lib.drb_packed_stride(2, 1, 3) == 16
    assert lib.drb_packed_stride(4, 3, 3) == -1
    ni, nl = C.c_int(), C.c_int()
    assert lib.drb_bvh_sizes(3, 262144, C.byref(ni), C.byref(nl)) == 0
    assert nl.value == 262144 * 33 and ni.value == nl.value - 1
    assert lib.drb_bvh_sizes(2, 6144, C.byref(ni), C.byref(nl)) == 0
    assert nl.value == 6144 * 17
    assert lib.drb_bvh_sizes(3, 0, C.byref(ni), C.byref(nl)) == 0
    assert nl.value == 2 and ni.value == 1
    assert lib.drb_bvh_sizes(3, 2 ** 27, C.byref(ni), C.byref(nl)) == L.DRB_ERR_INVALID_ARG
    assert b"too many" in lib.drb_last_error()


def test_invalid_arguments_rejected_without_gpu():
    from devil_ray_b200 import _lib as L
    lib = L.lib()
    m = L.DrbMesh()
    m.dim, m.order, m.ncomp, m.n_elem = 3, 7, 3, 1
    assert lib.drb_pack_elements(C.byref(m), None, None) == L.DRB_ERR_UNSUPPORTED
    assert lib.drb_radix_sort_pairs(None, None, None, None, -1, 30, None) == L.DRB_ERR_INVALID_ARG
    opts = L.DrbNewtonOpts(1e-4, 20, L.GUESS_GIVEN, None)
    m.order = 2
    b = L.DrbBvh()
    assert lib.drb_locate(C.byref(m), C.byref(b), None, 4, C.byref(opts), None, None,
                          L.DrbQueryStats(), None) == L.DRB_ERR_INVALID_ARG


def test_grid_rejects_missing_bvh():
    """drb_bvh_grid_size / drb_bvh_grid_build need a built BVH (no GPU use)."""
    import ctypes as C
    from devil_ray_b200 import _lib as L
    d = L.DrbBvh()
    m = C.c_longlong()
    assert L.lib().drb_bvh_grid_size(C.byref(d), 1.0, C.byref(m), None) == L.DRB_ERR_INVALID_ARG
    assert L.lib().drb_bvh_grid_build(C.byref(d), None) == L.DRB_ERR_INVALID_ARG
    assert L.lib().drb_bvh_grid_size(None, 1.0, C.byref(m), None) == L.DRB_ERR_INVALID_ARG


def test_widen_rejects_missing_bvh():
    from devil_ray_b200 import _lib as L
    lib = L.lib()
    assert lib.drb_bvh_widen(None, None, 0, None) == L.DRB_ERR_INVALID_ARG
    assert b"built BVH" in lib.drb_last_error()


def test_shape_queries_and_tet_rejections_without_gpu():
    """Dof counts, packed strides and reference-box sizes per element shape
    (tets, their triangle faces), and tets refused by a hex-only entry point
    before any GPU work."""
    from devil_ray_b200 import _lib as L
    lib = L.lib()
    T, S = L.SHAPE_TENSOR, L.SHAPE_SIMPLEX
    assert [lib.drb_elem_dofs(S, 3, p) for p in (1, 2, 3)] == [4, 10, 20]
    assert [lib.drb_elem_dofs(T, 3, p) for p in (1, 2, 3)] == [8, 27, 64]
    assert [lib.drb_elem_dofs(S, 2, p) for p in (1, 2, 3)] == [3, 6, 10]   # triangle faces
    assert lib.drb_elem_dofs(S, 3, 4) == -1
    assert [lib.drb_packed_stride_shape(S, 3, p, 3) for p in (1, 2, 3)] == [16, 36, 64]
    assert [lib.drb_packed_stride_shape(S, 3, p, 1) for p in (1, 2, 3)] == [4, 12, 20]
    assert lib.drb_packed_stride_shape(T, 3, 2, 3) == lib.drb_packed_stride(3, 2, 3)
    assert lib.drb_ref_box_floats(T, 3) == 6 and lib.drb_ref_box_floats(T, 2) == 4
    assert lib.drb_ref_box_floats(S, 3) == 12 and lib.drb_ref_box_floats(S, 2) == 6
    m = L.DrbMesh()
    m.dim, m.order, m.ncomp, m.n_elem, m.shape = 3, 2, 3, 1, S
    assert lib.drb_mesh_face_neighbors(C.byref(m), None, None) == L.DRB_ERR_INVALID_ARG
    assert b"hex" in lib.drb_last_error()
    m.shape = 7
    assert lib.drb_pack_elements(C.byref(m), None, None) == L.DRB_ERR_UNSUPPORTED
    m.dim, m.shape, m.n_elem = 2, S, 0
    assert lib.drb_pack_elements(C.byref(m), None, None) == L.DRB_OK   # triangle faces


def test_camera_moves_match_reference():
    """reset_to_bounds, elevate and azimuth give the reference Camera's
    position, look_at and field of view bit for bit."""
    import numpy as np
    from oracle import refpy
    from devil_ray_b200.render import Camera
    if not refpy.available():
        import pytest
        pytest.skip("reference oracle not built")
    cases = [((2.5, 2.5, 2.5), (0.5, 0.5, 0.5), None, (0, 0, 0), 10.0, 30.0),
             ((0.0, 0.0, 5.0), (0.0, 0.0, 0.0), (-1, 8, 0, 1, 0, 1), (0.1, 0.2, 0.0), 0.0, 0.0),
             ((3.0, -2.0, 1.0), (0.2, 0.1, -0.3), (-1, 1, -1, 1, -1, 1), (0.05, 0.0, 0.3),
              -25.0, 47.5),
             ((1.0, 2.0, 3.0), (0.0, 0.0, 0.0), (0, 1, 0, 2, 0, 0.5), (0, 0, 0), 89.0, -120.0)]
    for pos, look, bounds, pads, el, az in cases:
        c = Camera(320, 200, pos, look, (0.0, 1.0, 0.0), 30.0)
        if bounds is not None:
            c.reset_to_bounds(bounds, *pads)
        if el:
            c.elevate(el)
        if az:
            c.azimuth(az)
        cam9 = np.array([*pos, *look, 0.0, 1.0, 0.0], np.float32)
        want, fov = refpy.camera_move(320, 200, cam9, 30.0, bounds, pads, el, az)
        got = np.array([*c.pos, *c.look_at], np.float32)
        assert np.array_equal(got.view(np.uint32), want[:6].view(np.uint32)), (got, want[:6])
        assert np.float32(c.fov) == np.float32(fov)
