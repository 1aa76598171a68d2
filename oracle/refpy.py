"""Test oracle: ctypes wrapper over oracle/_ref/libdray_ref.so, the
reference's own C++ sources built by oracle/Makefile (see ref_api.cpp).

Test infrastructure only: imported by tests/, __graft_entry__.smoke() and the
bench's CPU-baseline leg, never by the product.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF_LIB = HERE / "_ref" / "libdray_ref.so"

_lib = None


def available() -> bool:
    return REF_LIB.exists()


def lib():
    global _lib
    if _lib is None:
        if not REF_LIB.exists():
            raise FileNotFoundError(f"{REF_LIB} not built (make -C oracle ref)")
        L = C.CDLL(str(REF_LIB))
        vp, ip, fp = C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_float)
        L.ref_last_error.restype = C.c_char_p
        L.ref_num_threads.restype = C.c_int
        L.ref_set_num_threads.argtypes = [C.c_int]
        L.ref_hex_create.restype = vp
        L.ref_hex_create.argtypes = [C.c_int, C.c_int, vp, C.c_int, vp, vp, C.c_int, vp]
        L.ref_free.argtypes = [vp]
        L.ref_bvh_sizes.argtypes = [vp, ip, ip]
        L.ref_bvh_copy.argtypes = [vp, vp, vp, vp, vp, vp]
        L.ref_morton.argtypes = [C.c_int, vp, vp, vp]
        L.ref_locate.argtypes = [vp, C.c_int, vp, vp, vp]
        L.ref_camera_rays.argtypes = [C.c_int, C.c_int, vp, C.c_float, vp]
        L.ref_volume.argtypes = [vp, C.c_int, C.c_int, vp, C.c_float, C.c_int, C.c_int, C.c_int,
                                 C.c_int, vp, C.c_int, vp, C.c_int, vp, vp, vp, C.c_int]
        L.ref_boundary.argtypes = [vp, vp, C.c_int]
        L.ref_surface.argtypes = [vp, C.c_int, C.c_int, vp, C.c_float, C.c_int, C.c_int, vp,
                                  C.c_int, vp, C.c_int, vp, vp, vp, vp, vp, vp]
        L.ref_eval_hex_scalar.argtypes = [C.c_int, C.c_int, vp, C.c_int, vp, vp, vp]
        L.ref_lineout.argtypes = [vp, C.c_int, vp, vp, C.c_int, C.c_float, vp, vp]
        L.ref_scalar_render.argtypes = [vp, C.c_int, C.c_int, vp, C.c_float, vp, vp, vp]
        L.ref_tri_create.restype = vp
        L.ref_tri_create.argtypes = [C.c_int, C.c_int, vp, C.c_int, vp, vp, C.c_int, vp]
        L.ref_quad_create.restype = vp
        L.ref_quad_create.argtypes = [C.c_int, C.c_int, vp, C.c_int, vp, vp, C.c_int, vp]
        L.ref_tet_create.restype = vp
        L.ref_tet_create.argtypes = [C.c_int, C.c_int, C.c_int, vp, C.c_int, vp, vp, C.c_int, vp]
        L.ref_eval_tet_scalar.argtypes = [C.c_int, C.c_int, vp, C.c_int, vp, vp, vp]
        L.ref_camera_move.argtypes = [C.c_int, C.c_int, vp, C.c_float, vp, vp, C.c_float,
                                      C.c_float, vp, vp]
        L.ref_render_scene.argtypes = [C.c_int, vp, vp, vp, vp, vp, vp, C.c_int, C.c_int, vp,
                                       C.c_float, vp, C.c_float, C.c_float, C.c_int, C.c_int,
                                       C.c_int, C.c_int, C.c_float, C.c_int, C.c_int, C.c_int,
                                       C.c_int, C.c_int, vp, C.c_int, vp, vp, vp, C.c_char_p]
        L.ref_hex_set_bvh.argtypes = [vp, C.c_int, vp, C.c_int, vp, vp, vp, vp]
        L.ref_volume_rays.argtypes = [vp, C.c_int, vp, C.c_int, C.c_int, C.c_int, C.c_int, vp,
                                      C.c_int, vp, C.c_int, vp, vp, C.c_int]
        _lib = L
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def set_threads(n: int):
    lib().ref_set_num_threads(int(n))


def num_threads() -> int:
    return lib().ref_num_threads()


class RefHexMesh:
    """The reference's UnstructuredMesh<Hex> (+ scalar field "f")."""

    def __init__(self, order, ctrl_idx, xyz, field=None):
        self.order = int(order)
        self.ctrl_idx = np.ascontiguousarray(ctrl_idx, dtype=np.int32)
        self.xyz = np.ascontiguousarray(xyz, dtype=np.float32).reshape(-1, 3)
        self.field = None if field is None else np.ascontiguousarray(field, dtype=np.float32)
        nd = (self.order + 1) ** 3
        self.n_elem = self.ctrl_idx.size // nd
        fptr = None if self.field is None else _p(self.field)
        self.h = lib().ref_hex_create(self.order, self.n_elem, _p(self.ctrl_idx), self.xyz.shape[0],
                                      _p(self.xyz), _p(self.ctrl_idx),
                                      0 if self.field is None else self.field.size, fptr)
        if not self.h:
            raise RuntimeError(lib().ref_last_error().decode())

    def __del__(self):
        if getattr(self, "h", None):
            lib().ref_free(self.h)
            self.h = None

    ref_box_floats = 6

    def bvh(self):
        ni, nl = C.c_int(), C.c_int()
        if lib().ref_bvh_sizes(self.h, C.byref(ni), C.byref(nl)) != 0:
            raise RuntimeError(lib().ref_last_error().decode())
        inner = np.zeros((ni.value, 16), np.float32)
        leaf = np.zeros(nl.value, np.int32)
        ids = np.zeros(nl.value, np.int32)
        bounds = np.zeros(6, np.float32)
        refb = np.zeros((nl.value, self.ref_box_floats), np.float32)
        if lib().ref_bvh_copy(self.h, _p(inner), _p(leaf), _p(ids), _p(bounds), _p(refb)) != 0:
            raise RuntimeError(lib().ref_last_error().decode())
        return {"inner": inner, "leaf_nodes": leaf, "aabb_ids": ids, "bounds": bounds,
                "ref_boxes": refb}

    def locate(self, pts):
        pts = np.ascontiguousarray(pts, dtype=np.float32).reshape(-1, 3)
        n = pts.shape[0]
        cell = np.zeros(n, np.int32)
        ref = np.zeros((n, 3), np.float32)
        if lib().ref_locate(self.h, n, _p(pts), _p(cell), _p(ref)) != 0:
            raise RuntimeError(lib().ref_last_error().decode())
        return cell, ref

    def set_bvh(self, inner, leaf_nodes, aabb_ids, bounds6, ref_boxes):
        """Install a BVH in the reference's record layout (inner [n,16],
        leaf element ids, leaf sub-box ids, bounds (xmin,xmax,...), reference
        boxes [n_leaf,6]) instead of the mesh's lazy build."""
        inner = np.ascontiguousarray(inner, np.float32).reshape(-1, 16)
        leaf = np.ascontiguousarray(leaf_nodes, np.int32)
        ids = np.ascontiguousarray(aabb_ids, np.int32)
        b6 = np.ascontiguousarray(bounds6, np.float32)
        rb = np.ascontiguousarray(ref_boxes, np.float32).reshape(-1, 6)
        if lib().ref_hex_set_bvh(self.h, inner.shape[0], _p(inner), leaf.size, _p(leaf), _p(ids),
                                 _p(b6), _p(rb)) != 0:
            raise RuntimeError(lib().ref_last_error().decode())

    def volume_rays(self, rays9, samples, use_lighting, tf_samples, rgb_pts, alpha_pts,
                    lights13):
        """Volume::integrate on the given rays (reference Ray records, 9
        floats each); returns the partials as (pixel, depth, r, g, b, a)."""
        rays = np.ascontiguousarray(rays9, np.float32).reshape(-1, 9)
        rgb = np.ascontiguousarray(rgb_pts, np.float32).reshape(-1)
        alp = np.ascontiguousarray(alpha_pts, np.float32).reshape(-1)
        lights = np.ascontiguousarray(lights13, np.float32).reshape(-1)
        maxp = 5 * rays.shape[0]
        parts = np.zeros((max(maxp, 1), 6), np.float32)
        n = lib().ref_volume_rays(self.h, rays.shape[0], _p(rays), samples, int(use_lighting),
                                  tf_samples, rgb.size // 4, _p(rgb), alp.size // 2, _p(alp),
                                  lights.size // 13, _p(lights), _p(parts), maxp)
        if n < 0:
            raise RuntimeError(lib().ref_last_error().decode())
        return parts[:n]

    def volume(self, w, h, cam9, fov, samples, use_lighting, tf_samples, rgb_pts, alpha_pts,
               lights13, want_partials=False):
        rgb = np.ascontiguousarray(rgb_pts, np.float32).reshape(-1)
        alp = np.ascontiguousarray(alpha_pts, np.float32).reshape(-1)
        lights = np.ascontiguousarray(lights13, np.float32).reshape(-1)
        cam = np.ascontiguousarray(cam9, np.float32)
        img = np.zeros((h, w, 4), np.float32)
        maxp = 5 * w * h if want_partials else 0
        parts = np.zeros((max(maxp, 1), 6), np.float32)
        n = lib().ref_volume(self.h, w, h, _p(cam), fov, samples, int(use_lighting), tf_samples,
                             rgb.size // 4, _p(rgb), alp.size // 2, _p(alp), lights.size // 13,
                             _p(lights), _p(img), _p(parts) if want_partials else None, maxp)
        if n < 0:
            raise RuntimeError(lib().ref_last_error().decode())
        return img, (parts[:n] if want_partials else None)

    def boundary_ctrl_idx(self):
        p = self.order
        maxf = 6 * self.n_elem
        out = np.zeros(maxf * (p + 1) ** 2, np.int32)
        nf = lib().ref_boundary(self.h, _p(out), maxf)
        if nf < 0:
            raise RuntimeError(lib().ref_last_error().decode())
        return out[: nf * (p + 1) ** 2].reshape(nf, (p + 1) ** 2)

    def scalar_render(self, w, h, cam9, fov):
        """ScalarRenderer::render's buffers on the boundary surface, field "f":
        (depth [h, w], zone id [h, w], scalar [h, w])."""
        cam = np.ascontiguousarray(cam9, np.float32)
        depth = np.zeros((h, w), np.float32)
        zone = np.zeros((h, w), np.int32)
        scal = np.zeros((h, w), np.float32)
        if lib().ref_scalar_render(self.h, w, h, _p(cam), fov, _p(depth), _p(zone), _p(scal)) < 0:
            raise RuntimeError(lib().ref_last_error().decode())
        return depth, zone, scal

    def lineout(self, starts, ends, samples, empty=0.0):
        """Lineout::execute on field "f": (points [n, 3], values [n])."""
        a = np.ascontiguousarray(starts, np.float32).reshape(-1, 3)
        b = np.ascontiguousarray(ends, np.float32).reshape(-1, 3)
        n = a.shape[0] * (samples + 2)
        pts = np.zeros((n, 3), np.float32)
        vals = np.zeros(n, np.float32)
        r = lib().ref_lineout(self.h, a.shape[0], _p(a), _p(b), samples, empty, _p(pts), _p(vals))
        if r < 0:
            raise RuntimeError(lib().ref_last_error().decode())
        return pts, vals

    def surface(self, w, h, cam9, fov, tf_samples, rgb_pts, alpha_pts, lights13):
        rgb = np.ascontiguousarray(rgb_pts, np.float32).reshape(-1)
        alp = np.ascontiguousarray(alpha_pts, np.float32).reshape(-1)
        lights = np.ascontiguousarray(lights13, np.float32).reshape(-1)
        cam = np.ascontiguousarray(cam9, np.float32)
        n = w * h
        hit = np.zeros(n, np.int32)
        dist = np.zeros(n, np.float32)
        ref2 = np.zeros((n, 2), np.float32)
        img = np.zeros((h, w, 4), np.float32)
        depth = np.zeros((h, w), np.float32)
        r = lib().ref_surface(self.h, w, h, _p(cam), fov, tf_samples, rgb.size // 4, _p(rgb),
                              alp.size // 2, _p(alp), lights.size // 13, _p(lights), _p(hit),
                              _p(dist), _p(ref2), _p(img), _p(depth))
        if r < 0:
            raise RuntimeError(lib().ref_last_error().decode())
        return {"hit_idx": hit, "dist": dist, "ref": ref2, "rgba": img, "depth": depth}


class RefTetMesh(RefHexMesh):
    """The reference's UnstructuredMesh<Tet> (+ scalar field "f"): the
    general-order element types, or with fixed=True the fixed-order P1/P2
    specialisations the reference's dispatcher also offers."""

    ref_box_floats = 12   # SubRef<3,Simplex>: u, v, w axis vertices, origin

    def __init__(self, order, ctrl_idx, xyz, field=None, fixed=False):
        self.order = int(order)
        self.ctrl_idx = np.ascontiguousarray(ctrl_idx, dtype=np.int32)
        self.xyz = np.ascontiguousarray(xyz, dtype=np.float32).reshape(-1, 3)
        self.field = None if field is None else np.ascontiguousarray(field, dtype=np.float32)
        nd = (self.order + 1) * (self.order + 2) * (self.order + 3) // 6
        self.n_elem = self.ctrl_idx.size // nd
        fptr = None if self.field is None else _p(self.field)
        self.h = lib().ref_tet_create(self.order, int(fixed), self.n_elem, _p(self.ctrl_idx),
                                      self.xyz.shape[0], _p(self.xyz), _p(self.ctrl_idx),
                                      0 if self.field is None else self.field.size, fptr)
        if not self.h:
            raise RuntimeError(lib().ref_last_error().decode())


class RefQuadMesh(RefHexMesh):
    """The reference's UnstructuredMesh<Quad> of a 2D mesh (+ scalar field "f")."""

    ref_box_floats = 4    # SubRef<2,Tensor>: low (u, v), high (u, v)

    def __init__(self, order, ctrl_idx, xyz, field=None):
        self.order = int(order)
        self.ctrl_idx = np.ascontiguousarray(ctrl_idx, dtype=np.int32)
        self.xyz = np.ascontiguousarray(xyz, dtype=np.float32).reshape(-1, 3)
        self.field = None if field is None else np.ascontiguousarray(field, dtype=np.float32)
        self.n_elem = self.ctrl_idx.size // ((self.order + 1) ** 2)
        fptr = None if self.field is None else _p(self.field)
        self.h = lib().ref_quad_create(self.order, self.n_elem, _p(self.ctrl_idx),
                                       self.xyz.shape[0], _p(self.xyz), _p(self.ctrl_idx),
                                       0 if self.field is None else self.field.size, fptr)
        if not self.h:
            raise RuntimeError(lib().ref_last_error().decode())


def _tet_boundary_ctrl_idx(self):
    p = self.order
    nd2 = (p + 1) * (p + 2) // 2
    maxf = 4 * self.n_elem
    out = np.zeros(maxf * nd2, np.int32)
    nf = lib().ref_boundary(self.h, _p(out), maxf)
    if nf < 0:
        raise RuntimeError(lib().ref_last_error().decode())
    return out[: nf * nd2].reshape(nf, nd2)


RefTetMesh.boundary_ctrl_idx = _tet_boundary_ctrl_idx


class RefTriMesh(RefHexMesh):
    """The reference's UnstructuredMesh<Tri> of a 2D mesh (+ scalar field "f")."""

    ref_box_floats = 6    # SubRef<2,Simplex>: u, v axis vertices, origin

    def __init__(self, order, ctrl_idx, xyz, field=None):
        self.order = int(order)
        self.ctrl_idx = np.ascontiguousarray(ctrl_idx, dtype=np.int32)
        self.xyz = np.ascontiguousarray(xyz, dtype=np.float32).reshape(-1, 3)
        self.field = None if field is None else np.ascontiguousarray(field, dtype=np.float32)
        self.n_elem = self.ctrl_idx.size // ((self.order + 1) * (self.order + 2) // 2)
        fptr = None if self.field is None else _p(self.field)
        self.h = lib().ref_tri_create(self.order, self.n_elem, _p(self.ctrl_idx),
                                      self.xyz.shape[0], _p(self.xyz), _p(self.ctrl_idx),
                                      0 if self.field is None else self.field.size, fptr)
        if not self.h:
            raise RuntimeError(lib().ref_last_error().decode())


def camera_move(w, h, cam9, fov, bounds6=None, pads=(0.0, 0.0, 0.0), elevate=0.0, azimuth=0.0):
    """The reference Camera after reset_to_bounds (when bounds6 is given),
    elevate and azimuth: (pos, look_at, up) as 9 floats, and the fov."""
    cam = np.ascontiguousarray(cam9, np.float32)
    out = np.zeros(9, np.float32)
    fov_out = np.zeros(1, np.float32)
    b6 = None if bounds6 is None else np.ascontiguousarray(bounds6, np.float32)
    p3 = np.ascontiguousarray(pads, np.float64)
    if lib().ref_camera_move(w, h, _p(cam), fov, None if b6 is None else _p(b6), _p(p3),
                             elevate, azimuth, _p(out), _p(fov_out)) != 0:
        raise RuntimeError(lib().ref_last_error().decode())
    return out, float(fov_out[0])


def render_scene(domains, w, h, cam9, fov, pads=None, elevate=0.0, azimuth=0.0, surface=True,
                 surface_domains=None, draw_mesh=False, line_thickness=0.05, volume=True, samples=200,
                 use_lighting=True, tf_samples=1024, rgb_pts=None, alpha_pts=None,
                 save_prefix=None):
    """The reference's Renderer::render over hex-mesh domains, each a tuple
    (order, ctrl_idx, xyz, field), the surface over the domain range
    surface_domains = (first, count) (all by default): returns (rgba [h, w,
    4], depth [h, w])."""
    sd = surface_domains if surface_domains is not None else (0, len(domains))
    orders = np.array([d[0] for d in domains], np.int32)
    nds = (orders + 1) ** 3
    n_el = np.array([np.asarray(d[1]).size // nd for d, nd in zip(domains, nds)], np.int32)
    n_ctrl = np.array([np.asarray(d[2]).reshape(-1, 3).shape[0] for d in domains], np.int32)
    ci = np.ascontiguousarray(np.concatenate([np.asarray(d[1], np.int32).ravel() for d in domains]))
    xyz = np.ascontiguousarray(np.concatenate([np.asarray(d[2], np.float32).ravel()
                                               for d in domains]))
    fld = np.ascontiguousarray(np.concatenate([np.asarray(d[3], np.float32).ravel()
                                               for d in domains]))
    rgb = np.ascontiguousarray(rgb_pts, np.float32).reshape(-1)
    alp = np.ascontiguousarray(alpha_pts, np.float32).reshape(-1)
    cam = np.ascontiguousarray(cam9, np.float32)
    p3 = None if pads is None else np.ascontiguousarray(pads, np.float64)
    rgba = np.zeros((h, w, 4), np.float32)
    depth = np.zeros((h, w), np.float32)
    st = lib().ref_render_scene(len(domains), _p(orders), _p(n_el), _p(n_ctrl), _p(ci), _p(xyz),
                                _p(fld), w, h, _p(cam), fov, None if p3 is None else _p(p3),
                                elevate, azimuth, int(surface), int(sd[0]), int(sd[1]),
                                int(draw_mesh), line_thickness,
                                int(volume), samples, int(use_lighting), tf_samples,
                                rgb.size // 4, _p(rgb), alp.size // 2, _p(alp), _p(rgba),
                                _p(depth),
                                None if save_prefix is None else str(save_prefix).encode())
    if st != 0:
        raise RuntimeError(lib().ref_last_error().decode())
    return rgba, depth


def eval_tet_scalar(p, vals, refs, fixed=False):
    """The reference's Element<3,1,Simplex,P>::eval_d of one scalar element."""
    vals = np.ascontiguousarray(vals, np.float32)
    refs = np.ascontiguousarray(refs, np.float32).reshape(-1, 3)
    n = refs.shape[0]
    v = np.zeros(n, np.float32)
    d = np.zeros((n, 3), np.float32)
    if lib().ref_eval_tet_scalar(p, int(fixed), _p(vals), n, _p(refs), _p(v), _p(d)) != 0:
        raise RuntimeError(lib().ref_last_error().decode())
    return v, d


def morton(aabbs6):
    a = np.ascontiguousarray(aabbs6, np.float32).reshape(-1, 6)
    codes = np.zeros(a.shape[0], np.uint32)
    bounds = np.zeros(6, np.float32)
    lib().ref_morton(a.shape[0], _p(a), _p(codes), _p(bounds))
    return codes, bounds


def camera_rays(w, h, cam9, fov):
    cam = np.ascontiguousarray(cam9, np.float32)
    rays = np.zeros((w * h, 9), np.float32)
    n = lib().ref_camera_rays(w, h, _p(cam), fov, _p(rays))
    if n < 0:
        raise RuntimeError(lib().ref_last_error().decode())
    return rays


def eval_hex_scalar(p, vals, refs, fixed=False):
    """The reference's Element<3,1,Tensor,P>::eval_d of one scalar element."""
    vals = np.ascontiguousarray(vals, np.float32)
    refs = np.ascontiguousarray(refs, np.float32).reshape(-1, 3)
    n = refs.shape[0]
    v = np.zeros(n, np.float32)
    d = np.zeros((n, 3), np.float32)
    if lib().ref_eval_hex_scalar(p, int(fixed), _p(vals), n, _p(refs), _p(v), _p(d)) != 0:
        raise RuntimeError(lib().ref_last_error().decode())
    return v, d
