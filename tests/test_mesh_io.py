"""Readers of order-1 meshes (devil_ray_b200.mesh_io), on the host.

* the MFEM ASCII reader on a small hand-written beam and on the reference's
  own test meshes (when the reference checkout is present), which must
  reproduce the committed fixture arrays the GPU tests use;
* the BlueprintLowOrder::import semantics (io/blueprint_low_order.cpp):
  uniform, structured and explicit topologies, the per-shape corner maps,
  vertex and element fields, and the errors the reference raises;
* the fixture meshes through the reference's own locate (oracle/_ref):
  every element's centroid is found in that element.
"""
import hashlib
import os
from pathlib import Path

import numpy as np
import pytest

from devil_ray_b200 import mesh_io

FIXTURE = Path(__file__).resolve().parent / "golden" / "mfem_order1_meshes.npz"
# the reference checkout's test data, read only to pin the fixture arrays
REF_DATA = Path(os.environ.get("DRB_REF_SRC", "/root/reference/src")) / "tests" / "dray" / "data"

BEAM2 = """MFEM mesh v1.0
# two unit cubes along x
dimension
3

elements
2
1 5 0 1 4 3 6 7 10 9
2 5 1 2 5 4 7 8 11 10

boundary
0

vertices
12
3
0 0 0
1 0 0
2 0 0
0 1 0
1 1 0
2 1 0
0 0 1
1 0 1
2 0 1
0 1 1
1 1 1
2 1 1
"""


def test_mfem_reader_hex_lexicographic_order():
    m = mesh_io.read_mfem_mesh(BEAM2)
    assert m.shape == "hex" and m.n_elem == 2 and m.dim == 3
    c = m.ctrl_idx.reshape(2, 8)
    # lexicographic (x fastest, z slowest) corners of each cube
    lex = np.array([[i, j, k] for k in (0, 1) for j in (0, 1) for i in (0, 1)], np.float32)
    for e in range(2):
        assert np.array_equal(m.xyz[c[e]] - m.xyz[c[e, 0]], lex)
    assert np.array_equal(m.fields["attribute"].values, [1.0, 2.0])


def test_mfem_reader_rejects_bad_input():
    with pytest.raises(ValueError):
        mesh_io.read_mfem_mesh("MFEM mesh v1.1\ndimension\n3\n")
    bad = BEAM2.replace("1 5 0 1 4 3 6 7 10 9", "1 5 0 1 4 3 6 7 10 99")
    with pytest.raises(ValueError, match="outside"):
        mesh_io.read_mfem_mesh(bad)
    mixed = BEAM2.replace("2 5 1 2 5 4 7 8 11 10", "2 4 1 2 5 4")
    with pytest.raises(ValueError, match="geometries"):
        mesh_io.read_mfem_mesh(mixed)
    curved = BEAM2.replace("vertices\n12\n3\n", "vertices\n12\n\nnodes\nFiniteElementSpace\n")
    with pytest.raises(ValueError, match="nodes"):
        mesh_io.read_mfem_mesh(curved)


def test_fixture_matches_reference_files():
    """The committed fixture arrays are what the reader makes of the
    reference's files (skipped where the checkout is absent)."""
    if not REF_DATA.exists():
        pytest.skip("reference checkout not present")
    fx = np.load(FIXTURE)
    for name in ("beam-hex", "fichera", "beam-tet", "beam-quad", "beam-tri"):
        path = REF_DATA / f"{name}.mesh"
        assert str(fx[f"{name}/sha256"]) == hashlib.sha256(path.read_bytes()).hexdigest()
        m = mesh_io.read_mfem_mesh(path)
        assert str(fx[f"{name}/shape"]) == m.shape
        assert np.array_equal(fx[f"{name}/ctrl_idx"], m.ctrl_idx)
        assert np.array_equal(fx[f"{name}/xyz"], m.xyz)


def test_blueprint_uniform_and_structured():
    node = {"coordsets": {"c": {"type": "uniform", "dims": {"i": 3, "j": 3, "k": 3},
                                "origin": {"x": -1.0, "y": 0.0, "z": 2.0},
                                "spacing": {"dx": 0.5, "dy": 1.0, "dz": 2.0}}},
            "topologies": {"t": {"type": "uniform", "coordset": "c"}},
            "fields": {"f": {"topology": "t", "association": "vertex",
                             "values": np.arange(27.0)},
                       "e": {"topology": "t", "association": "element",
                             "values": np.arange(8.0)}}}
    (m,) = mesh_io.import_low_order(node)
    assert m.shape == "hex" and m.n_elem == 8 and m.xyz.shape == (27, 3)
    assert np.allclose(m.xyz[1], [-0.5, 0.0, 2.0]) and np.allclose(m.xyz[26], [0.0, 2.0, 6.0])
    c = m.ctrl_idx.reshape(8, 8)
    # cell (1, 0, 1): first corner (1, 0, 1) = 1 + 9, then +x, +y, +x+y, then +z
    assert np.array_equal(c[5], [10, 11, 13, 14, 19, 20, 22, 23])
    assert m.fields["f"].order == 1 and np.array_equal(m.fields["f"].ctrl_idx, m.ctrl_idx)
    assert m.fields["e"].order == 0
    ci, v = m.fields["e"].as_order1("hex")
    assert ci.size == 64 and np.array_equal(v.reshape(8, 8)[3], np.full(8, 3.0))
    # the same grid as a structured topology over explicit coordinates
    x, y, z = (m.xyz[:, k] for k in range(3))
    snode = {"coordsets": {"c": {"type": "explicit", "values": {"x": x, "y": y, "z": z}}},
             "topologies": {"t": {"type": "structured", "coordset": "c",
                                  "elements": {"dims": {"i": 2, "j": 2, "k": 2}}}}}
    (s,) = mesh_io.import_low_order(snode)
    assert np.array_equal(s.ctrl_idx, m.ctrl_idx) and np.array_equal(s.xyz, m.xyz)
    # 2D uniform: quads with z = 0
    n2 = {"coordsets": {"c": {"type": "uniform", "dims": {"i": 4, "j": 2}}},
          "topologies": {"t": {"type": "uniform", "coordset": "c"}}}
    (q,) = mesh_io.import_low_order(n2)
    assert q.shape == "quad" and q.n_elem == 3
    assert np.array_equal(q.ctrl_idx.reshape(3, 4)[2], [2, 3, 6, 7])
    assert np.all(q.xyz[:, 2] == 0)


def test_blueprint_explicit_corner_maps():
    """convert_conn: out[dof] = in[map[dof]] with the reference's maps."""
    xyz = np.random.default_rng(0).random((12, 3))
    node = {"coordsets": {"c": {"type": "explicit",
                                "values": {"x": xyz[:, 0], "y": xyz[:, 1], "z": xyz[:, 2]}}},
            "topologies": {"t": {"type": "unstructured", "coordset": "c",
                                 "elements": {"shape": "hex",
                                              "connectivity": np.arange(8, dtype=np.int64)}}}}
    (m,) = mesh_io.import_low_order(node)
    assert np.array_equal(m.ctrl_idx, [0, 1, 4, 5, 3, 2, 7, 6])
    assert m.xyz.dtype == np.float32
    for shape, conn, want in (("quad", [5, 6, 7, 8], [5, 6, 8, 7]),
                              ("tet", [1, 2, 3, 4], [1, 2, 3, 4]),
                              ("tri", [9, 10, 11], [9, 10, 11])):
        node["topologies"]["t"]["elements"] = {"shape": shape,
                                               "connectivity": np.array(conn, np.int32)}
        (m,) = mesh_io.import_low_order(node)
        assert m.shape == shape and np.array_equal(m.ctrl_idx, want)
    node["topologies"]["t"]["elements"] = {"shape": "wedge", "connectivity": np.arange(6)}
    with pytest.raises(ValueError, match="not currently supported"):
        mesh_io.import_low_order(node)
    node["topologies"]["t"]["elements"] = {"shape": "hex",
                                           "connectivity": np.arange(8, dtype=np.float32)}
    with pytest.raises(ValueError, match="conn data type"):
        mesh_io.import_low_order(node)
    node["topologies"]["t"] = {"type": "rectilinear", "coordset": "c"}
    with pytest.raises(ValueError, match="not implemented"):
        mesh_io.import_low_order(node)


@pytest.mark.parametrize("name", ["beam-hex", "fichera", "beam-tet", "beam-quad", "beam-tri"])
def test_reference_locates_fixture_centroids(ref, name):
    """Every element's vertex centroid lies in that element: the reference's
    locate returns the element with an inside reference point."""
    fx = np.load(FIXTURE)
    shape = str(fx[f"{name}/shape"])
    ci, xyz = fx[f"{name}/ctrl_idx"], fx[f"{name}/xyz"]
    nd = mesh_io.DOFS[shape]
    cen = xyz[ci.reshape(-1, nd)].mean(axis=1).astype(np.float32)
    if shape == "hex":
        r = ref.RefHexMesh(1, ci, xyz)
    elif shape == "tet":
        r = ref.RefTetMesh(1, ci, xyz)
    elif shape == "quad":
        r = ref.RefQuadMesh(1, ci, xyz)
    else:
        r = ref.RefTriMesh(1, ci, xyz)
    cell, rr = r.locate(cen)
    assert np.array_equal(cell, np.arange(cen.shape[0]))
    dims = 3 if shape in ("hex", "tet") else 2
    assert np.all(rr[:, :dims] > 0.0) and np.all(rr[:, :dims] < 1.0)
