"""ctypes binding of the C-ABI in include/drb.h (libdrb.so, built in-tree).

The library is loaded from the package directory only; there is no CPU
fallback.  If the shared object is missing the import fails loudly.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

_PKG = Path(__file__).resolve().parent
LIB_PATH = _PKG / "libdrb.so"

DRB_OK = 0
DRB_ERR_INVALID_ARG = 1
DRB_ERR_OOM = 2
DRB_ERR_CUDA = 3
DRB_ERR_QUEUE_GIVEUP = 4
DRB_ERR_UNSUPPORTED = 5

GUESS_ZERO = 0
GUESS_ELEM_CENTER = 1
GUESS_SUBREF_CENTER = 2
GUESS_GIVEN = 3
GUESS_SUBBOX_LINEAR = 4

SHAPE_TENSOR = 0
SHAPE_SIMPLEX = 1


class DrbMesh(C.Structure):
    _fields_ = [("dim", C.c_int), ("order", C.c_int), ("ncomp", C.c_int),
                ("n_elem", C.c_int), ("n_ctrl", C.c_int),
                ("ctrl_idx", C.c_void_p), ("values", C.c_void_p), ("packed", C.c_void_p),
                ("face_neighbors", C.c_void_p), ("shape", C.c_int),
                ("hull_planes", C.c_void_p)]


class DrbBvh(C.Structure):
    _fields_ = [("n_inner", C.c_int), ("n_leaf", C.c_int),
                ("inner_nodes", C.c_void_p), ("leaf_nodes", C.c_void_p),
                ("aabb_ids", C.c_void_p), ("ref_boxes", C.c_void_p),
                ("bounds", C.c_float * 6), ("wide_nodes", C.c_void_p), ("n_wide", C.c_int),
                ("wide_depth", C.c_int), ("leaf_maps", C.c_void_p),
                ("grid_start", C.c_void_p), ("grid_entries", C.c_void_p),
                ("grid_boxes", C.c_void_p),
                ("grid_dims", C.c_int * 3), ("grid_origin", C.c_float * 3),
                ("grid_inv", C.c_float * 3)]


class DrbNewtonOpts(C.Structure):
    _fields_ = [("tol", C.c_float), ("max_steps", C.c_int), ("guess_mode", C.c_int),
                ("guess", C.c_void_p)]


class DrbQueryStats(C.Structure):
    _fields_ = [("iters", C.c_void_p), ("candidates", C.c_void_p), ("nodes", C.c_void_p)]


class DrbLocateConfig(C.Structure):
    _fields_ = [("block", C.c_int), ("blocks_per_sm", C.c_int), ("chunk", C.c_int),
                ("sort_queries", C.c_int), ("reg_elements", C.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class DrbCamera(C.Structure):
    _fields_ = [("width", C.c_int), ("height", C.c_int), ("pos", C.c_float * 3),
                ("look_at", C.c_float * 3), ("up", C.c_float * 3), ("fov_y", C.c_float),
                ("zoom", C.c_float)]


class DrbRayStats(C.Structure):
    _fields_ = [("samples", C.c_void_p), ("iters", C.c_void_p), ("candidates", C.c_void_p)]


class DrbVolumeOpts(C.Structure):
    _fields_ = [("samples", C.c_int), ("use_lighting", C.c_int), ("tol", C.c_float),
                ("max_steps", C.c_int), ("guess_mode", C.c_int), ("coherent", C.c_int),
                ("bounds", C.c_float * 6), ("cull", C.c_int)]


class DrbError(RuntimeError):
    def __init__(self, status: int, where: str, msg: str):
        super().__init__(f"{where} failed with status {status}: {msg}")
        self.status = status


_lib = None

# name -> (restype, argtypes)
_SIGS = {
    "drb_last_error": (C.c_char_p, []),
    "drb_version": (C.c_int, []),
    "drb_noalloc_max_queries": (C.c_int, []),
    "drb_locate_batched_noalloc": (C.c_int, [C.POINTER(DrbMesh), C.POINTER(DrbBvh), C.c_void_p,
                                             C.c_int, C.POINTER(DrbNewtonOpts), C.c_void_p,
                                             C.c_void_p, C.c_void_p, DrbQueryStats,
                                             C.c_void_p]),
    "drb_mesh_boundary": (C.c_int, [C.POINTER(DrbMesh), C.c_void_p, C.c_void_p, C.c_void_p,
                                    C.c_void_p, C.POINTER(C.c_int), C.c_void_p]),
    "drb_surface_intersect": (C.c_int, [C.POINTER(DrbMesh), C.POINTER(DrbBvh), C.c_void_p,
                                        C.c_int, C.c_float, C.c_int, C.c_void_p, DrbRayStats,
                                        C.c_void_p]),
    "drb_surface_shade": (C.c_int, [C.POINTER(DrbMesh), C.POINTER(DrbMesh), C.c_void_p,
                                    C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p,
                                    C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                                    C.c_void_p, C.c_void_p]),
    "drb_ray_max": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]),
    "drb_camera_rays": (C.c_int, [C.POINTER(DrbCamera), C.c_void_p, C.c_void_p]),
    "drb_default_light": (C.c_int, [C.POINTER(DrbCamera), C.c_void_p]),
    "drb_camera_elevate": (C.c_int, [C.POINTER(DrbCamera), C.c_float]),
    "drb_camera_azimuth": (C.c_int, [C.POINTER(DrbCamera), C.c_float]),
    "drb_camera_reset_to_bounds": (C.c_int, [C.POINTER(DrbCamera), C.c_void_p, C.c_double,
                                             C.c_double, C.c_double]),
    "drb_cull_rays": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p,
                                C.POINTER(C.c_int), C.c_void_p]),
    "drb_field_range": (C.c_int, [C.POINTER(DrbMesh), C.c_void_p, C.c_void_p]),
    "drb_color_table_sample": (C.c_int, [C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_int,
                                         C.c_int, C.c_float, C.c_float, C.c_void_p]),
    "drb_volume_integrate": (C.c_int, [C.POINTER(DrbMesh), C.POINTER(DrbMesh), C.POINTER(DrbBvh),
                                       C.c_void_p, C.c_int, C.POINTER(DrbVolumeOpts), C.c_void_p,
                                       C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p,
                                       C.POINTER(C.c_int), DrbRayStats, C.c_void_p]),
    "drb_volume_render": (C.c_int, [C.POINTER(DrbMesh), C.POINTER(DrbMesh), C.POINTER(DrbBvh),
                                    C.c_void_p, C.c_int, C.POINTER(DrbVolumeOpts), C.c_void_p,
                                    C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p,
                                    C.c_void_p, DrbRayStats, C.c_void_p]),
    "drb_composite_partials": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
    "drb_framebuffer_clear": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
    "drb_framebuffer_composite_background": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p,
                                                       C.c_void_p]),
    "drb_kernel_launches": (C.c_ulonglong, []),
    "drb_locate_batched": (C.c_int, [C.POINTER(DrbMesh), C.POINTER(DrbBvh), C.c_void_p, C.c_int,
                                     C.POINTER(DrbNewtonOpts), C.c_void_p, C.c_void_p,
                                     C.c_void_p, DrbQueryStats, C.c_void_p]),
    "drb_query_order": (C.c_int, [C.POINTER(DrbBvh), C.c_void_p, C.c_int, C.c_void_p,
                                  C.c_void_p]),
    "drb_bvh_leaf_maps": (C.c_int, [C.POINTER(DrbMesh), C.POINTER(DrbBvh), C.c_void_p,
                                    C.c_void_p]),
    "drb_bvh_grid_size": (C.c_int, [C.POINTER(DrbBvh), C.c_float, C.POINTER(C.c_longlong),
                                    C.c_void_p]),
    "drb_bvh_grid_build": (C.c_int, [C.POINTER(DrbBvh), C.c_void_p]),
    "drb_query_stage": (C.c_int, [C.POINTER(DrbBvh), C.c_void_p, C.c_int, C.c_void_p,
                                  C.c_void_p]),
    "drb_locate_staged": (C.c_int, [C.POINTER(DrbMesh), C.POINTER(DrbBvh), C.c_void_p, C.c_int,
                                    C.POINTER(DrbNewtonOpts), C.c_void_p, C.c_void_p,
                                    C.c_void_p, C.c_void_p, DrbQueryStats, C.c_void_p]),
    "drb_locate_ordered": (C.c_int, [C.POINTER(DrbMesh), C.POINTER(DrbBvh), C.c_void_p, C.c_int,
                                     C.c_void_p, C.POINTER(DrbNewtonOpts), C.c_void_p,
                                     C.c_void_p, C.c_void_p, DrbQueryStats, C.c_void_p]),
    "drb_locate_host": (C.c_int, [C.POINTER(DrbMesh), C.POINTER(DrbBvh), C.c_void_p, C.c_int,
                                  C.POINTER(DrbNewtonOpts), C.c_void_p, C.c_int, C.c_void_p,
                                  C.c_void_p, C.c_void_p]),
    "drb_locate_tune": (C.c_int, [C.POINTER(DrbMesh), C.POINTER(DrbBvh), C.c_void_p, C.c_int,
                                  C.POINTER(DrbNewtonOpts), C.c_void_p, C.POINTER(C.c_float),
                                  C.c_void_p]),
    "drb_packed_stride": (C.c_int, [C.c_int, C.c_int, C.c_int]),
    "drb_elem_dofs": (C.c_int, [C.c_int, C.c_int, C.c_int]),
    "drb_packed_stride_shape": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int]),
    "drb_ref_box_floats": (C.c_int, [C.c_int, C.c_int]),
    "drb_tet_hull_planes": (C.c_int, [C.POINTER(DrbMesh), C.c_void_p, C.c_void_p]),
    "drb_pack_elements": (C.c_int, [C.POINTER(DrbMesh), C.c_void_p, C.c_void_p]),
    "drb_bvh_sizes": (C.c_int, [C.c_int, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "drb_elem_subboxes": (C.c_int, [C.POINTER(DrbMesh), C.c_void_p, C.c_void_p, C.c_void_p,
                                    C.c_void_p, C.c_void_p]),
    "drb_morton_codes": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]),
    "drb_radix_sort_pairs": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                       C.c_int, C.c_int, C.c_void_p]),
    "drb_lbvh_build": (C.c_int, [C.POINTER(DrbMesh), C.POINTER(DrbBvh), C.c_void_p, C.c_void_p]),
    "drb_scalar_buffer_write": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int,
                                          C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "drb_lineout_points": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p,
                                     C.c_void_p]),
    "drb_field_eval": (C.c_int, [C.POINTER(DrbMesh), C.c_void_p, C.c_void_p, C.c_int, C.c_float,
                                 C.c_void_p, C.c_void_p]),
    "drb_mesh_face_neighbors": (C.c_int, [C.POINTER(DrbMesh), C.c_void_p, C.c_void_p]),
    "drb_bvh_widen": (C.c_int, [C.POINTER(DrbBvh), C.c_void_p, C.c_int, C.c_void_p]),
    "drb_locate": (C.c_int, [C.POINTER(DrbMesh), C.POINTER(DrbBvh), C.c_void_p, C.c_int,
                             C.POINTER(DrbNewtonOpts), C.c_void_p, C.c_void_p, DrbQueryStats,
                             C.c_void_p]),
}


def declared_symbols():
    """Names of every entry point declared in include/drb.h."""
    import re
    hdr = (_PKG.parent / "include" / "drb.h").read_text()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(drb_\w+)\s*\(", hdr, re.M)))


def lib():
    """Load libdrb.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} is missing: run __graft_entry__.build() "
                              "(no CPU fallback exists)")
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in _SIGS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(status: int, where: str):
    if status != DRB_OK:
        raise DrbError(status, where, lib().drb_last_error().decode(errors="replace"))
