"""Readers of non-synthetic order-1 meshes into the path's data layout.

Two sources, both producing order-1 Bernstein geometry (for order-1
elements the control points are the vertices):

* ``import_low_order(node)``: the semantics of the reference's
  ``BlueprintLowOrder::import`` (io/blueprint_low_order.cpp:610-1050) over a
  plain nested dict laid out like a Conduit Blueprint mesh node
  (``coordsets``, ``topologies``, ``fields``).  Uniform, structured and
  unstructured (explicit) topologies; hex, quad, tet and tri shapes; vertex
  fields become order-1 fields over the topology's connectivity, element
  fields order-0 fields over a counting index, as in the reference.
  Explicit connectivity is reordered per element by the reference's maps
  (io/blueprint_low_order.cpp:22-25): ``out[dof] = in[map[dof]]`` with the
  hex map 0,1,4,5,3,2,7,6.  Structured and uniform topologies use the
  reference's lexicographic corner order (x fastest;
  io/blueprint_low_order.cpp:257-328).

* ``read_mfem_mesh(path)``: MFEM's ASCII ``MFEM mesh v1.0`` format without a
  ``nodes`` section (order-1 geometry: the vertices are the control points).
  The reference reads these files through MFEM (io/mfem_reader.cpp,
  mfem2dray.cpp:835-960), which maps MFEM's element dofs into the
  lexicographic order (x inner, z outer) with the H1 element's dof map; for
  order 1 that is corners 0,1,3,2,4,5,7,6 of MFEM's hex and 0,1,3,2 of its
  quad, and the identity for tets and triangles (mfem2dray.cpp:30-170).

Both return ``LowOrderMesh`` records whose ``ctrl_idx`` / ``xyz`` arrays feed
``api.UnstructuredMesh`` and the reference's ``GridFunction`` unchanged.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

# BlueprintLowOrder's per-element reorderings (io/blueprint_low_order.cpp:22-25)
BLUEPRINT_CONN_MAP = {
    "hex": (0, 1, 4, 5, 3, 2, 7, 6),
    "quad": (0, 1, 3, 2),
    "tet": (0, 1, 2, 3),
    "tri": (0, 1, 2),
}
# MFEM order-1 corner order -> lexicographic dof order
MFEM_LEX_MAP = {
    "hex": (0, 1, 3, 2, 4, 5, 7, 6),
    "quad": (0, 1, 3, 2),
    "tet": (0, 1, 2, 3),
    "tri": (0, 1, 2),
}
# MFEM geometry ids (mesh/geom.hpp) of the element kinds on the path
MFEM_GEOMETRY = {2: "tri", 3: "quad", 4: "tet", 5: "hex"}
DOFS = {"hex": 8, "quad": 4, "tet": 4, "tri": 3}
DIM = {"hex": 3, "tet": 3, "quad": 2, "tri": 2}


@dataclass
class LowOrderField:
    """A scalar field: order 1 (vertex values over the mesh's connectivity)
    or order 0 (one value per element)."""
    name: str
    order: int
    ctrl_idx: np.ndarray
    values: np.ndarray

    def as_order1(self, shape: str) -> tuple[np.ndarray, np.ndarray]:
        """(ctrl_idx, values) of an order-1 field with the same values: an
        order-0 field becomes a constant over each element, with its own
        control points per element (exact: equal Bernstein coefficients
        reproduce the constant)."""
        if self.order == 1:
            return self.ctrl_idx, self.values
        nd = DOFS[shape]
        n = self.values.shape[0]
        return (np.arange(n * nd, dtype=np.int32),
                np.repeat(self.values.astype(np.float32), nd))


@dataclass
class LowOrderMesh:
    shape: str                      # "hex", "quad", "tet" or "tri"
    ctrl_idx: np.ndarray            # int32 [n_elem * dofs]
    xyz: np.ndarray                 # float32 [n_ctrl, 3] (z = 0 for 2D input)
    order: int = 1
    name: str = "mesh"
    fields: dict = field(default_factory=dict)

    @property
    def dim(self) -> int:
        return DIM[self.shape]

    @property
    def n_elem(self) -> int:
        return self.ctrl_idx.size // DOFS[self.shape]

    @property
    def simplex(self) -> bool:
        return self.shape in ("tet", "tri")

    def device_mesh(self, device="cuda"):
        """The path's mesh object (api.UnstructuredMesh) over these arrays."""
        from . import _lib as L
        from . import api
        return api.UnstructuredMesh(self.ctrl_idx, self.xyz, 1, dim=self.dim, device=device,
                                    shape=L.SHAPE_SIMPLEX if self.simplex else L.SHAPE_TENSOR)


# ---------------------------------------------------------------- blueprint

def _coords_explicit(n_coords) -> np.ndarray:
    """import_explicit_coords (io/blueprint_low_order.cpp:167-235): x, y and
    an optional z (0 when absent), as float32."""
    v = n_coords["values"]
    x = np.asarray(v["x"], np.float64)
    y = np.asarray(v["y"], np.float64)
    z = np.asarray(v["z"], np.float64) if "z" in v else np.zeros_like(x)
    if not (x.shape == y.shape == z.shape):
        raise ValueError("coordset: x, y and z differ in length")
    return np.stack([x, y, z], axis=1).astype(np.float32)


def structured_conn(point_dims, is_3d: bool) -> np.ndarray:
    """structured_conn (io/blueprint_low_order.cpp:257-328): lexicographic
    corners (x fastest) of every cell of a logically structured grid."""
    nx, ny = int(point_dims[0]), int(point_dims[1])
    nz = int(point_dims[2]) if is_3d else 1
    cx, cy, cz = nx - 1, ny - 1, max(nz - 1, 1)
    if cx < 1 or cy < 1 or (is_3d and nz < 2):
        raise ValueError("structured topology needs at least one cell per axis")
    i = np.arange(cx)
    j = np.arange(cy)
    if not is_3d:
        jj, ii = np.meshgrid(j, i, indexing="ij")
        c0 = (jj * nx + ii).ravel()
        return np.stack([c0, c0 + 1, c0 + nx, c0 + nx + 1], axis=1).astype(np.int32).ravel()
    k = np.arange(cz)
    kk, jj, ii = np.meshgrid(k, j, i, indexing="ij")
    c0 = ((kk * ny + jj) * nx + ii).ravel()
    c4 = c0 + nx * ny
    return np.stack([c0, c0 + 1, c0 + nx, c0 + nx + 1, c4, c4 + 1, c4 + nx, c4 + nx + 1],
                    axis=1).astype(np.int32).ravel()


def _import_uniform(n_coords):
    """BlueprintLowOrder::import_uniform (io/blueprint_low_order.cpp:920-1048)."""
    if n_coords.get("type") != "uniform":
        raise ValueError("uniform topology needs a uniform coordset")
    d = n_coords["dims"]
    is_2d = "k" not in d
    dims = (int(d["i"]), int(d["j"]), 1 if is_2d else int(d["k"]))
    o = n_coords.get("origin", {})
    s = n_coords.get("spacing", {})
    ox, oy, oz = (float(o.get(a, 0.0)) for a in ("x", "y", "z"))
    sx, sy, sz = (float(s.get(a, 1.0)) for a in ("dx", "dy", "dz"))
    kk, jj, ii = np.meshgrid(np.arange(dims[2]), np.arange(dims[1]), np.arange(dims[0]),
                             indexing="ij")
    x = ox + ii.ravel() * sx
    y = oy + jj.ravel() * sy
    z = np.zeros_like(x) if is_2d else oz + kk.ravel() * sz
    xyz = np.stack([x, y, z], axis=1).astype(np.float32)
    shape = "quad" if is_2d else "hex"
    return shape, structured_conn(dims, not is_2d), xyz


def _import_structured(n_coords, n_topo):
    """BlueprintLowOrder::import_structured (io/blueprint_low_order.cpp:749-815)."""
    xyz = _coords_explicit(n_coords)
    e = n_topo["elements"]["dims"]
    is_3d = "k" in e
    dims = (int(e["i"]) + 1, int(e["j"]) + 1, int(e["k"]) + 1 if is_3d else 1)
    if dims[0] * dims[1] * dims[2] != xyz.shape[0]:
        raise ValueError("structured topology: dims do not match the coordset")
    return ("hex" if is_3d else "quad"), structured_conn(dims, is_3d), xyz


def _import_explicit(n_coords, n_topo):
    """BlueprintLowOrder::import_explicit (io/blueprint_low_order.cpp:817-918)
    with convert_conn's per-element reordering (:47-74)."""
    if n_coords.get("type") != "explicit":
        raise ValueError("unstructured topology needs an explicit coordset")
    xyz = _coords_explicit(n_coords)
    shape = n_topo["elements"]["shape"]
    if shape not in BLUEPRINT_CONN_MAP:
        raise ValueError(f"Shape '{shape}' not currently supported")
    conn = np.asarray(n_topo["elements"]["connectivity"])
    if conn.dtype.kind not in "iu":
        raise ValueError("Unsupported conn data type")
    nd = DOFS[shape]
    if conn.size % nd:
        raise ValueError(f"connectivity length {conn.size} is not a multiple of {nd}")
    conn = conn.reshape(-1, nd)[:, list(BLUEPRINT_CONN_MAP[shape])]
    if conn.size and (conn.min() < 0 or conn.max() >= xyz.shape[0]):
        raise ValueError("connectivity refers to a vertex outside the coordset")
    return shape, conn.astype(np.int32).ravel(), xyz


def import_low_order(node: dict) -> list[LowOrderMesh]:
    """BlueprintLowOrder::import over a dict Blueprint node: one
    LowOrderMesh per topology, each with the scalar fields on it."""
    meshes = {}
    topos = node.get("topologies", {})
    if not topos:
        raise ValueError("Import failed to verify: no topologies")
    for name, n_topo in topos.items():
        n_coords = node["coordsets"][n_topo["coordset"]]
        kind = n_topo["type"]
        if kind == "uniform":
            shape, conn, xyz = _import_uniform(n_coords)
        elif kind == "unstructured":
            shape, conn, xyz = _import_explicit(n_coords, n_topo)
        elif kind == "structured":
            shape, conn, xyz = _import_structured(n_coords, n_topo)
        else:
            raise ValueError(f"not implemented {kind}")
        meshes[name] = LowOrderMesh(shape, conn, xyz, 1, name)
    for fname, n_field in node.get("fields", {}).items():
        m = meshes[n_field["topology"]]
        vals = n_field["values"]
        if isinstance(vals, dict):
            if len(vals) != 1:
                raise ValueError(f"fields with {len(vals)} components are not supported here")
            vals = next(iter(vals.values()))
        vals = np.asarray(vals, np.float32).ravel()
        if n_field["association"] == "vertex":
            if vals.size != m.xyz.shape[0]:
                raise ValueError(f"field {fname}: {vals.size} values for {m.xyz.shape[0]} vertices")
            m.fields[fname] = LowOrderField(fname, 1, m.ctrl_idx, vals)
        else:
            if vals.size != m.n_elem:
                raise ValueError(f"field {fname}: {vals.size} values for {m.n_elem} elements")
            m.fields[fname] = LowOrderField(fname, 0, np.arange(m.n_elem, dtype=np.int32), vals)
    return list(meshes.values())


# --------------------------------------------------------------------- mfem

def _tokens(text: str):
    for line in text.splitlines():
        line = line.split("#", 1)[0].strip()
        if line:
            yield line


def read_mfem_mesh(source) -> LowOrderMesh:
    """An ``MFEM mesh v1.0`` file (path or text) with order-1 geometry."""
    text = Path(source).read_text() if not (isinstance(source, str) and "\n" in source) \
        else source
    lines = list(_tokens(text))
    if not lines or not lines[0].startswith("MFEM mesh v1.0"):
        raise ValueError("not an 'MFEM mesh v1.0' file")
    pos = 1
    dim = None
    elements = None
    xyz = None
    while pos < len(lines):
        key = lines[pos]
        pos += 1
        if key == "dimension":
            dim = int(lines[pos])
            pos += 1
        elif key == "elements":
            n = int(lines[pos])
            pos += 1
            elements = [tuple(int(t) for t in lines[pos + e].split()) for e in range(n)]
            pos += n
        elif key == "boundary":
            n = int(lines[pos])
            pos += 1 + n
        elif key == "vertices":
            n = int(lines[pos])
            pos += 1
            if pos < len(lines) and lines[pos].startswith("nodes"):
                raise ValueError("curved (nodes) MFEM meshes need MFEM's finite element spaces")
            vdim = int(lines[pos])
            pos += 1
            v = np.array([[float(t) for t in lines[pos + i].split()] for i in range(n)],
                         np.float64).reshape(n, vdim)
            pos += n
            xyz = np.zeros((n, 3), np.float32)
            xyz[:, :vdim] = v
        elif key == "nodes" or key.startswith("FiniteElement"):
            raise ValueError("curved (nodes) MFEM meshes need MFEM's finite element spaces")
        elif key == "mfem_mesh_end":
            break
        else:
            raise ValueError(f"unsupported MFEM mesh section '{key}'")
    if dim is None or elements is None or xyz is None:
        raise ValueError("MFEM mesh without dimension, elements or vertices")
    geoms = {e[1] for e in elements}
    if len(geoms) != 1 or next(iter(geoms)) not in MFEM_GEOMETRY:
        raise ValueError(f"mixed or unsupported MFEM element geometries {sorted(geoms)}")
    shape = MFEM_GEOMETRY[next(iter(geoms))]
    if DIM[shape] != dim:
        raise ValueError(f"{shape} elements in a dimension-{dim} mesh")
    nd = DOFS[shape]
    conn = np.array([e[2:] for e in elements], np.int64)
    if conn.shape[1] != nd:
        raise ValueError("element vertex count does not match its geometry")
    conn = conn[:, list(MFEM_LEX_MAP[shape])]
    if conn.min() < 0 or conn.max() >= xyz.shape[0]:
        raise ValueError("element refers to a vertex outside the vertex list")
    attrs = np.array([e[0] for e in elements], np.int32)
    m = LowOrderMesh(shape, conn.astype(np.int32).ravel(), xyz, 1,
                     Path(source).stem if not (isinstance(source, str) and "\n" in source)
                     else "mesh")
    m.fields["attribute"] = LowOrderField("attribute", 0, np.arange(len(elements), dtype=np.int32),
                                          attrs.astype(np.float32))
    return m
