"""Seeded synthetic Bernstein hex meshes and query sets for the benchmark
workloads.

Lattice convention (the reference's synthetic generators,
synthetic/affine_radial.cpp:124-139,193-240): a mesh of n^3 elements of
order p shares one lattice of (p*n+1)^3 control points, point (I,J,K) at
flat index (K*(p*n+1)+J)*(p*n+1)+I; element (ei,ej,ek) has id
(ek*n+ej)*n+ei and its dof (a,b,c) (u fastest) is lattice point
(p*ei+a, p*ej+b, p*ek+c).  The same ctrl_idx serves the geometry and the
scalar field.

Workloads (sizes and distributions; all randomness from numpy PCG64 with a
recorded seed):
  volume_8     8^3 hex P2, interior points displaced by
               0.05*sin(2pi x)sin(2pi y)sin(2pi z) on every axis,
               f = sin(3x)cos(2y)+z^2 at the displaced control point
  surface_32   32^3 hex P3, same warp with amplitude 0.08 plus uniform +-0.01
               jitter per interior control point
  locate_64    64^3 hex P2 whose geometry is exactly trilinear per element:
               the vertex lattice is displaced by uniform offsets up to
               `distortion` x h (boundary vertices keep their normal
               coordinate) and the P2 control points interpolate the
               element corners
  volume_128   128^3 hex P3, warp 0.05, f = sum of 8 seeded Gaussians
               (sigma 0.1)
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

TWO_PI = 2.0 * np.pi


@dataclass
class HexMeshData:
    order: int
    n: int                      # elements per axis
    ctrl_idx: np.ndarray        # int32 [n_elem * (p+1)^3]
    xyz: np.ndarray             # float32 [n_ctrl, 3]
    field: np.ndarray           # float32 [n_ctrl]
    meta: dict = field(default_factory=dict)

    @property
    def n_elem(self) -> int:
        return self.n ** 3

    @property
    def n_ctrl(self) -> int:
        return self.xyz.shape[0]

    @property
    def nd(self) -> int:
        return (self.order + 1) ** 3


def lattice_ctrl_idx(n: int, p: int) -> np.ndarray:
    """ctrl_idx of an n^3 order-p hex lattice mesh (element-major, u fastest)."""
    m = p * n + 1
    e = np.arange(n, dtype=np.int64)
    a = np.arange(p + 1, dtype=np.int64)
    # element (ek, ej, ei), dof (c, b, a) -> lattice (p*ek+c, p*ej+b, p*ei+a)
    K = (p * e[:, None, None, None, None, None] + a[None, None, None, :, None, None])
    J = (p * e[None, :, None, None, None, None] + a[None, None, None, None, :, None])
    I = (p * e[None, None, :, None, None, None] + a[None, None, None, None, None, :])
    idx = (K * m + J) * m + I
    return idx.reshape(-1).astype(np.int32)


def lattice_points(n: int, p: int) -> np.ndarray:
    """Undisplaced lattice coordinates in [0,1]^3, float64 [m^3, 3]."""
    m = p * n + 1
    t = np.linspace(0.0, 1.0, m)
    Z, Y, X = np.meshgrid(t, t, t, indexing="ij")
    return np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)


def interior_mask(n: int, p: int) -> np.ndarray:
    m = p * n + 1
    i = np.arange(m)
    inner = (i > 0) & (i < m - 1)
    Z, Y, X = np.meshgrid(inner, inner, inner, indexing="ij")
    return (X & Y & Z).ravel()


def field_sincos(xyz: np.ndarray) -> np.ndarray:
    x, y, z = xyz[:, 0], xyz[:, 1], xyz[:, 2]
    return np.sin(3.0 * x) * np.cos(2.0 * y) + z * z


def field_gaussians(xyz: np.ndarray, seed: int, count: int = 8, sigma: float = 0.1):
    rng = np.random.default_rng(seed)
    centres = rng.uniform(0.15, 0.85, size=(count, 3))
    amps = rng.uniform(0.5, 1.0, size=count)
    f = np.zeros(xyz.shape[0], dtype=np.float64)
    for c, a in zip(centres, amps):
        d2 = ((xyz - c) ** 2).sum(axis=1)
        f += a * np.exp(-d2 / (2.0 * sigma * sigma))
    return f, centres, amps


def warped_mesh(n: int, p: int, amp: float, jitter: float = 0.0, seed: int = 0,
                gaussian_field_seed: int | None = None) -> HexMeshData:
    base = lattice_points(n, p)
    inner = interior_mask(n, p)
    s = np.sin(TWO_PI * base[:, 0]) * np.sin(TWO_PI * base[:, 1]) * np.sin(TWO_PI * base[:, 2])
    disp = amp * s
    xyz = base.copy()
    xyz[inner] += disp[inner, None]
    if jitter > 0.0:
        rng = np.random.default_rng(seed)
        j = rng.uniform(-jitter, jitter, size=(int(inner.sum()), 3))
        xyz[inner] += j
    meta = {"warp_amplitude": amp, "jitter": jitter, "seed": seed}
    if gaussian_field_seed is None:
        f = field_sincos(xyz)
        meta["field"] = "sin(3x)cos(2y)+z^2"
    else:
        f, c, a = field_gaussians(xyz, gaussian_field_seed)
        meta["field"] = "8 gaussians sigma 0.1"
        meta["field_seed"] = gaussian_field_seed
    return HexMeshData(order=p, n=n, ctrl_idx=lattice_ctrl_idx(n, p),
                       xyz=xyz.astype(np.float32), field=f.astype(np.float32), meta=meta)


def trilinear_distorted_mesh(n: int, p: int, distortion: float, seed: int) -> HexMeshData:
    """Order-p mesh whose elements are trilinear maps of a randomly displaced
    vertex lattice (offsets uniform in [-distortion*h, distortion*h] per axis,
    boundary vertices keep the coordinate normal to their boundary plane)."""
    h = 1.0 / n
    t = np.linspace(0.0, 1.0, n + 1)
    Z, Y, X = np.meshgrid(t, t, t, indexing="ij")
    verts = np.stack([X, Y, Z], axis=-1)           # [k, j, i, 3]
    rng = np.random.default_rng(seed)
    off = rng.uniform(-distortion * h, distortion * h, size=verts.shape)
    idx = np.arange(n + 1)
    on_b = (idx == 0) | (idx == n)
    off[..., 0] *= ~on_b[None, None, :]
    off[..., 1] *= ~on_b[None, :, None]
    off[..., 2] *= ~on_b[:, None, None]
    verts = verts + off
    m = p * n + 1
    L = np.arange(m)
    e = np.minimum(L // p, n - 1)
    u = (L - p * e) / p                             # 0, 1/p, ..., 1
    ek, ej, ei = np.meshgrid(e, e, e, indexing="ij")
    w, v, uu = np.meshgrid(u, u, u, indexing="ij")
    xyz = np.zeros((m, m, m, 3))
    for c in range(2):
        for b in range(2):
            for a in range(2):
                wt = ((uu if a else 1 - uu) * (v if b else 1 - v) * (w if c else 1 - w))
                xyz += wt[..., None] * verts[ek + c, ej + b, ei + a]
    xyz = xyz.reshape(-1, 3)
    f = field_sincos(xyz)
    meta = {"distortion": distortion, "seed": seed, "field": "sin(3x)cos(2y)+z^2"}
    return HexMeshData(order=p, n=n, ctrl_idx=lattice_ctrl_idx(n, p),
                       xyz=xyz.astype(np.float32), field=f.astype(np.float32), meta=meta)


@dataclass
class TetMeshData:
    order: int
    n: int                      # cubes per axis (6 tets each)
    ctrl_idx: np.ndarray        # int32 [n_elem * (p+1)(p+2)(p+3)/6]
    xyz: np.ndarray             # float32 [n_ctrl, 3]
    field: np.ndarray           # float32 [n_ctrl]
    meta: dict = field(default_factory=dict)

    @property
    def n_elem(self) -> int:
        return 6 * self.n ** 3

    @property
    def n_ctrl(self) -> int:
        return self.xyz.shape[0]

    @property
    def nd(self) -> int:
        return tet_dofs(self.order)


def tet_dofs(p: int) -> int:
    return (p + 1) * (p + 2) * (p + 3) // 6


def tet_multi_indices(p: int):
    """Dof multi-indices (i, j, k) of an order-p tet in the reference's dof
    order: i (power of u) fastest, then j (v), then k (w)."""
    return [(i, j, k) for k in range(p + 1) for j in range(p + 1 - k) for i in range(p + 1 - k - j)]


# The six tets of a cube (Kuhn subdivision): for a permutation (a, b, c) of
# the axes, vertices v0 = cube origin, v1 = v0 + e_a, v2 = v1 + e_b,
# v3 = v2 + e_c.  Every cube uses the same diagonal, so faces match.
KUHN_PERMS = ((0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0))


def tet_lattice_ctrl_idx(n: int, p: int) -> np.ndarray:
    """ctrl_idx of the 6 n^3 order-p tets of an n^3 cube lattice over the
    (p n + 1)^3 lattice points of lattice_points(n, p).  Tet (cube c, perm
    q) has id 6 * ((ck n + cj) n + ci) + q; its reference vertices are
    origin -> v0, u = 1 -> v1, v = 1 -> v2, w = 1 -> v3, so dof (i, j, k)
    sits at lattice point p v0 + i e_a + j (e_a + e_b) + k (e_a + e_b + e_c)."""
    m = p * n + 1
    mi = np.array(tet_multi_indices(p), np.int64)             # [nd, 3]
    out = np.empty((n, n, n, 6, mi.shape[0]), np.int64)
    c = np.arange(n, dtype=np.int64)
    CK, CJ, CI = np.meshgrid(c, c, c, indexing="ij")
    for q, (a, b, cc) in enumerate(KUHN_PERMS):
        off = np.zeros((mi.shape[0], 3), np.int64)            # lattice offset (x, y, z)
        off[:, a] += mi[:, 0] + mi[:, 1] + mi[:, 2]
        off[:, b] += mi[:, 1] + mi[:, 2]
        off[:, cc] += mi[:, 2]
        X = p * CI[..., None] + off[None, None, None, :, 0]
        Y = p * CJ[..., None] + off[None, None, None, :, 1]
        Z = p * CK[..., None] + off[None, None, None, :, 2]
        out[:, :, :, q, :] = (Z * m + Y) * m + X
    return out.reshape(-1).astype(np.int32)


def tet_warped_mesh(n: int, p: int, amp: float, jitter: float = 0.0, seed: int = 0) -> TetMeshData:
    """6 n^3 order-p tets filling [0,1]^3, interior lattice points displaced
    by amp * sin(2pi x) sin(2pi y) sin(2pi z) on every axis (plus optional
    uniform jitter), f = sin(3x)cos(2y)+z^2 at the displaced points."""
    base = lattice_points(n, p)
    inner = interior_mask(n, p)
    s = np.sin(TWO_PI * base[:, 0]) * np.sin(TWO_PI * base[:, 1]) * np.sin(TWO_PI * base[:, 2])
    xyz = base.copy()
    xyz[inner] += (amp * s)[inner, None]
    if jitter > 0.0:
        rng = np.random.default_rng(seed)
        xyz[inner] += rng.uniform(-jitter, jitter, size=(int(inner.sum()), 3))
    meta = {"warp_amplitude": amp, "jitter": jitter, "seed": seed,
            "field": "sin(3x)cos(2y)+z^2", "cells": "6 Kuhn tets per cube"}
    return TetMeshData(order=p, n=n, ctrl_idx=tet_lattice_ctrl_idx(n, p),
                       xyz=xyz.astype(np.float32), field=field_sincos(xyz).astype(np.float32),
                       meta=meta)


@dataclass
class QuadMeshData:
    order: int
    n: int                      # quads per axis
    ctrl_idx: np.ndarray        # int32 [n^2 * (p+1)^2], u fastest
    xyz: np.ndarray             # float32 [(p n + 1)^2, 3], z = 0
    field: np.ndarray           # float32 [n_ctrl]
    meta: dict = field(default_factory=dict)

    @property
    def n_elem(self) -> int:
        return self.n ** 2


def quad_warped_mesh(n: int, p: int, amp: float, jitter: float = 0.0, seed: int = 0) -> QuadMeshData:
    """A 2D mesh of n^2 order-p quads over [0,1]^2 in the z = 0 plane:
    lattice (p n + 1)^2, point (I, J) at index J (p n + 1) + I, element
    (ei, ej) with id ej n + ei and dof (a, b) (u fastest) at lattice point
    (p ei + a, p ej + b); interior points displaced by
    amp sin(2pi x) sin(2pi y) in x and y (plus optional uniform jitter);
    f = sin(3x)cos(2y) + x y."""
    m = p * n + 1
    t = np.linspace(0.0, 1.0, m)
    Y, X = np.meshgrid(t, t, indexing="ij")
    xyz = np.stack([X.ravel(), Y.ravel(), np.zeros(m * m)], axis=1)
    i = np.arange(m)
    inner1 = (i > 0) & (i < m - 1)
    inner = (inner1[:, None] & inner1[None, :]).ravel()
    s = np.sin(TWO_PI * xyz[:, 0]) * np.sin(TWO_PI * xyz[:, 1])
    xyz[inner, :2] += (amp * s)[inner, None]
    if jitter > 0.0:
        rng = np.random.default_rng(seed)
        xyz[inner, :2] += rng.uniform(-jitter, jitter, size=(int(inner.sum()), 2))
    e = np.arange(n, dtype=np.int64)
    a = np.arange(p + 1, dtype=np.int64)
    J = p * e[:, None, None, None] + a[None, None, :, None]
    I = p * e[None, :, None, None] + a[None, None, None, :]
    idx = (J * m + I).reshape(-1).astype(np.int32)
    f = np.sin(3.0 * xyz[:, 0]) * np.cos(2.0 * xyz[:, 1]) + xyz[:, 0] * xyz[:, 1]
    meta = {"warp_amplitude": amp, "jitter": jitter, "seed": seed, "field": "sin(3x)cos(2y)+xy"}
    return QuadMeshData(order=p, n=n, ctrl_idx=idx, xyz=xyz.astype(np.float32),
                        field=f.astype(np.float32), meta=meta)


def tri_warped_mesh(n: int, p: int, amp: float, jitter: float = 0.0, seed: int = 0) -> QuadMeshData:
    """The lattice of quad_warped_mesh(n, p, ...) cut into 2 n^2 order-p
    triangles along each cell's (0,0)-(1,1) diagonal.  Triangle 2 c of cell
    c has vertices (0,0), (1,0), (1,1) (origin, u = 1, v = 1), triangle
    2 c + 1 has (0,0), (1,1), (0,1); dof (i, j) (i fastest) sits at lattice
    offset (i + j, j) and (i, i + j) respectively."""
    q = quad_warped_mesh(n, p, amp, jitter, seed)
    m = p * n + 1
    mi = [(i, j) for j in range(p + 1) for i in range(p + 1 - j)]
    off0 = np.array([(i + j, j) for i, j in mi], np.int64)        # (dx, dy)
    off1 = np.array([(i, i + j) for i, j in mi], np.int64)
    c = np.arange(n, dtype=np.int64)
    CJ, CI = np.meshgrid(c, c, indexing="ij")
    out = np.empty((n, n, 2, len(mi)), np.int64)
    for t, off in enumerate((off0, off1)):
        X = p * CI[..., None] + off[None, None, :, 0]
        Y = p * CJ[..., None] + off[None, None, :, 1]
        out[:, :, t, :] = Y * m + X
    meta = dict(q.meta)
    meta["cells"] = "2 triangles per square"
    return QuadMeshData(order=p, n=n, ctrl_idx=out.reshape(-1).astype(np.int32), xyz=q.xyz,
                        field=q.field, meta=meta)


# outside fraction of uniform queries: the meshes fill [0,1]^3, so queries are
# drawn from a cube padded so that about 8% of its volume lies outside
OUTSIDE_FRACTION = 0.08
QUERY_PAD = ((1.0 / (1.0 - OUTSIDE_FRACTION)) ** (1.0 / 3.0) - 1.0) / 2.0


def uniform_queries(count: int, seed: int, pad: float = QUERY_PAD) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return rng.uniform(-pad, 1.0 + pad, size=(count, 3)).astype(np.float32)


def workload_mesh(name: str) -> HexMeshData:
    if name == "volume_8":
        return warped_mesh(8, 2, 0.05)
    if name == "surface_32":
        return warped_mesh(32, 3, 0.08, jitter=0.01, seed=1)
    if name == "locate_64":
        return trilinear_distorted_mesh(64, 2, 0.15, seed=2)
    if name == "locate_64_d25":
        return trilinear_distorted_mesh(64, 2, 0.25, seed=3)
    if name == "volume_128":
        return warped_mesh(128, 3, 0.05, gaussian_field_seed=4)
    raise KeyError(name)


# Camera and transfer function of the volume/surface workloads
CAMERA = {"pos": (2.5, 2.5, 2.5), "look_at": (0.5, 0.5, 0.5), "up": (0.0, 1.0, 0.0),
          "fov": 30.0}
TF_RGB = [(0.0, 0.23, 0.30, 0.75), (1.0, 0.71, 0.02, 0.15)]   # (pos, r, g, b)
TF_ALPHA = [(0.0, 0.05), (1.0, 0.9)]                            # (pos, alpha)
