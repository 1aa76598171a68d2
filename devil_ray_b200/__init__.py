"""devil_ray_b200: B200-native (sm_100a) ray-element hot path of Devil Ray.

LBVH over Bernstein element sub-boxes, BVH traversal, Newton inversion of
order 1-3 hex/quad elements, field evaluation and compositing, behind a
C-ABI (include/drb.h, libdrb.so) with a host mirror of the reference's
data model.  No CPU fallback: the CUDA library must be built.
"""
from ._lib import lib, LIB_PATH  # noqa: F401

__all__ = ["lib", "LIB_PATH"]
