"""Host-side mirror of the reference's data model for this path, over the
C-ABI (libdrb.so), with torch tensors as device-memory plumbing.

Names follow Devil Ray (src/dray):
  GridFunction        data_model/grid_function.hpp:19-50
  UnstructuredMesh    data_model/unstructured_mesh.hpp (get_bvh, locate, bounds)
  UnstructuredField   data_model/unstructured_field.hpp
  BVH                 bvh.hpp:16-37
  Location            location.hpp:16-20 (cell id, reference point)

All compute goes through libdrb.so; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib as L


def _ptr(t: torch.Tensor | None):
    if t is None:
        return None
    return C.c_void_p(t.data_ptr())


def _stream(stream=None):
    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)


def _dev(a, dtype, device):
    if isinstance(a, torch.Tensor):
        return a.to(device=device, dtype=dtype).contiguous()
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device=device).contiguous()


@dataclass
class GridFunction:
    """ctrl_idx int32[n_elem*nd] + values float[n_ctrl, ncomp] on the device."""
    ctrl_idx: torch.Tensor
    values: torch.Tensor
    el_dofs: int

    @property
    def num_elem(self) -> int:
        return self.ctrl_idx.numel() // self.el_dofs


class BVH:
    """Device BVH in the reference layout (4 x float4 per inner node)."""

    def __init__(self, dim: int, n_elem: int, device, shape: int = L.SHAPE_TENSOR):
        ni, nl = C.c_int(), C.c_int()
        L.check(L.lib().drb_bvh_sizes(dim, n_elem, C.byref(ni), C.byref(nl)), "drb_bvh_sizes")
        self.n_inner, self.n_leaf = ni.value, nl.value
        self.inner_nodes = torch.empty((self.n_inner, 16), dtype=torch.float32, device=device)
        self.leaf_nodes = torch.empty(self.n_leaf, dtype=torch.int32, device=device)
        self.aabb_ids = torch.empty(self.n_leaf, dtype=torch.int32, device=device)
        rbf = L.lib().drb_ref_box_floats(shape, dim)
        self.ref_boxes = torch.empty((self.n_leaf, rbf), dtype=torch.float32, device=device)
        self.bounds = np.zeros(6, np.float32)
        self.sorted_codes = None
        # optional 4-wide traversal tree (drb_bvh_widen)
        self.wide_nodes = None
        self.n_wide = 0
        self.wide_depth = 0
        # optional per-leaf linear maps (drb_bvh_leaf_maps)
        self.leaf_maps = None
        # optional uniform-grid candidate lists (drb_bvh_grid_build)
        self.grid_start = None
        self.grid_entries = None
        self.grid_boxes = None
        self.grid_geom = None  # (dims, origin, inv)

    def desc(self) -> L.DrbBvh:
        d = L.DrbBvh()
        d.n_inner, d.n_leaf = self.n_inner, self.n_leaf
        d.inner_nodes = self.inner_nodes.data_ptr()
        d.leaf_nodes = self.leaf_nodes.data_ptr()
        d.aabb_ids = self.aabb_ids.data_ptr()
        d.ref_boxes = self.ref_boxes.data_ptr()
        for q in range(6):
            d.bounds[q] = float(self.bounds[q])
        if self.wide_nodes is not None:
            d.wide_nodes = self.wide_nodes.data_ptr()
            d.n_wide, d.wide_depth = self.n_wide, self.wide_depth
        if self.leaf_maps is not None:
            d.leaf_maps = self.leaf_maps.data_ptr()
        if self.grid_start is not None:
            d.grid_start = self.grid_start.data_ptr()
            d.grid_entries = self.grid_entries.data_ptr()
            d.grid_boxes = self.grid_boxes.data_ptr()
            dims, origin, inv = self.grid_geom
            for q in range(3):
                d.grid_dims[q], d.grid_origin[q], d.grid_inv[q] = dims[q], origin[q], inv[q]
        return d

    def build_grid(self, cell_scale: float = 1.0, stream=None):
        """Uniform-grid candidate lists of the leaves (drb_bvh_grid_size +
        drb_bvh_grid_build): the batched locates then scan the point's cell
        instead of walking the tree, with identical candidates and results.
        Cells are about cell_scale times the mean leaf extent per axis."""
        self.grid_start = self.grid_entries = self.grid_boxes = self.grid_geom = None
        d = self.desc()
        m = C.c_longlong()
        L.check(L.lib().drb_bvh_grid_size(C.byref(d), float(cell_scale), C.byref(m),
                                          _stream(stream)), "drb_bvh_grid_size")
        dims = tuple(d.grid_dims)
        dev = self.inner_nodes.device
        self.grid_start = torch.empty(dims[0] * dims[1] * dims[2] + 1, dtype=torch.int32,
                                      device=dev)
        self.grid_entries = torch.empty(m.value, dtype=torch.int32, device=dev)
        self.grid_boxes = torch.empty((self.n_leaf, 8), dtype=torch.float32, device=dev)
        self.grid_geom = (dims, tuple(d.grid_origin), tuple(d.grid_inv))
        d = self.desc()
        L.check(L.lib().drb_bvh_grid_build(C.byref(d), _stream(stream)), "drb_bvh_grid_build")
        return self


    def build_leaf_maps(self, mesh: "UnstructuredMesh", stream=None):
        """Per-leaf linear maps of the element maps at the reference
        sub-box centres (drb_bvh_leaf_maps), for GUESS_SUBBOX_LINEAR."""
        maps = torch.empty((self.n_leaf, 16), dtype=torch.float32,
                           device=self.inner_nodes.device)
        L.check(L.lib().drb_bvh_leaf_maps(C.byref(mesh.desc()), C.byref(self.desc()),
                                          _ptr(maps), _stream(stream)), "drb_bvh_leaf_maps")
        self.leaf_maps = maps
        return self

    def widen(self, stream=None):
        """Build the 4-wide traversal tree of this BVH (same candidates in
        the same order; one 128-byte node per two binary levels)."""
        d = self.desc()
        L.check(L.lib().drb_bvh_widen(C.byref(d), None, 0, _stream(stream)), "drb_bvh_widen")
        self.wide_nodes = torch.empty((max(d.n_wide, 1), 32), dtype=torch.float32,
                                      device=self.inner_nodes.device)
        L.check(L.lib().drb_bvh_widen(C.byref(d), _ptr(self.wide_nodes), d.n_wide,
                                      _stream(stream)), "drb_bvh_widen")
        self.n_wide, self.wide_depth = d.n_wide, d.wide_depth
        return self

    def binary_only(self) -> "BVH":
        """A view of the same BVH without the wide tree (the binary traversal)."""
        b = BVH.__new__(BVH)
        b.__dict__.update(self.__dict__)
        b.wide_nodes, b.n_wide, b.wide_depth = None, 0, 0
        b.grid_start = b.grid_entries = b.grid_boxes = b.grid_geom = None
        return b

    def without_grid(self) -> "BVH":
        """A view of the same BVH without its grid lists (tree traversal)."""
        b = BVH.__new__(BVH)
        b.__dict__.update(self.__dict__)
        b.grid_start = b.grid_entries = b.grid_boxes = b.grid_geom = None
        return b


class UnstructuredMesh:
    """Bernstein mesh of order 1..3: tensor hex (dim 3) or quad (dim 2)
    elements, or with shape=SHAPE_SIMPLEX tets (dim 3) - the reference's
    UnstructuredMesh<Hex*/Quad*/Tet*> (data_model/unstructured_mesh.hpp)."""

    def __init__(self, ctrl_idx, xyz, order: int, dim: int = 3, device="cuda", pack: bool = True,
                 shape: int = L.SHAPE_TENSOR):
        self.dim = dim
        self.order = int(order)
        self.shape = int(shape)
        nd = L.lib().drb_elem_dofs(self.shape, dim, self.order)
        if nd < 0:
            raise ValueError(f"unsupported mesh: shape {shape}, dim {dim}, order {order}")
        self.dof_data = GridFunction(_dev(ctrl_idx, torch.int32, device),
                                     _dev(xyz, torch.float32, device).reshape(-1, 3), nd)
        self.device = torch.device(device)
        self.packed = None
        self._neighbors = None
        self._hull = None
        self._bvh = None
        if pack:
            self.pack()

    @property
    def n_elem(self) -> int:
        return self.dof_data.num_elem

    def cells(self) -> int:
        return self.n_elem

    def desc(self, packed: bool = True) -> L.DrbMesh:
        m = L.DrbMesh()
        m.dim, m.order, m.ncomp = self.dim, self.order, 3
        m.shape = self.shape
        m.n_elem = self.n_elem
        m.n_ctrl = self.dof_data.values.shape[0]
        m.ctrl_idx = self.dof_data.ctrl_idx.data_ptr()
        m.values = self.dof_data.values.data_ptr()
        m.packed = self.packed.data_ptr() if (packed and self.packed is not None) else None
        nb = getattr(self, "_neighbors", None)
        m.face_neighbors = nb.data_ptr() if nb is not None else None
        hp = getattr(self, "_hull", None)
        m.hull_planes = hp.data_ptr() if hp is not None else None
        return m

    def face_neighbors(self, stream=None):
        """Element across each face of every element (six per hex, four per
        tet; -1 on the boundary), built once (drb_mesh_face_neighbors); the
        volume march follows rays across faces with it."""
        if getattr(self, "_neighbors", None) is None:
            fpe = 4 if self.shape == L.SHAPE_SIMPLEX else 6
            nb = torch.empty((max(self.n_elem, 1), fpe), dtype=torch.int32, device=self.device)
            d = self.desc()
            L.check(L.lib().drb_mesh_face_neighbors(C.byref(d), _ptr(nb), _stream(stream)),
                    "drb_mesh_face_neighbors")
            self._neighbors = nb
        return self._neighbors

    def hull_planes(self, stream=None):
        """Tets: the bounding planes of every element (drb_tet_hull_planes),
        built once; the batched locate filters its candidates with them."""
        if self._hull is None and self.shape == L.SHAPE_SIMPLEX and self.dim == 3:
            hp = torch.empty((max(self.n_elem, 1), 20), dtype=torch.float32, device=self.device)
            d = self.desc()
            L.check(L.lib().drb_tet_hull_planes(C.byref(d), _ptr(hp), _stream(stream)),
                    "drb_tet_hull_planes")
            self._hull = hp
        return self._hull

    def pack(self, stream=None):
        stride = L.lib().drb_packed_stride_shape(self.shape, self.dim, self.order, 3)
        self.packed = torch.empty((max(self.n_elem, 1), stride), dtype=torch.float32,
                                  device=self.device)
        d = self.desc(packed=False)
        L.check(L.lib().drb_pack_elements(C.byref(d), _ptr(self.packed), _stream(stream)),
                "drb_pack_elements")

    def get_bvh(self, stream=None, keep_codes: bool = False) -> BVH:
        """Lazily build the LBVH (UnstructuredMesh::get_bvh,
        data_model/unstructured_mesh.cpp:23-31) and its 4-wide traversal
        tree."""
        if self._bvh is None:
            self._bvh = self.build_bvh(stream, keep_codes)
            self._bvh.widen(stream)
            if self.shape == L.SHAPE_SIMPLEX and self.dim == 3:
                self.hull_planes(stream)
        return self._bvh

    def build_bvh(self, stream=None, keep_codes: bool = False) -> BVH:
        b = BVH(self.dim, self.n_elem, self.device, self.shape)
        codes = None
        if keep_codes:
            codes = torch.empty(b.n_leaf, dtype=torch.int32, device=self.device)
        d = self.desc()
        bd = b.desc()
        L.check(L.lib().drb_lbvh_build(C.byref(d), C.byref(bd), _ptr(codes), _stream(stream)),
                "drb_lbvh_build")
        b.bounds = np.array(list(bd.bounds), np.float32)
        b.sorted_codes = codes
        return b

    def bounds(self):
        return self.get_bvh().bounds

    def locate(self, points, tol: float = 1e-4, max_steps: int = 20,
               guess_mode: int = L.GUESS_ELEM_CENTER, guess=None, stats: bool = False,
               stream=None, packed: bool = True):
        """Mesh::locate: returns (cell int32[n], ref float[n,3]) and, with
        stats=True, (iterations, candidates) per point."""
        pts = _dev(points, torch.float32, self.device).reshape(-1, 3)
        n = pts.shape[0]
        cell = torch.empty(n, dtype=torch.int32, device=self.device)
        ref = torch.empty((n, 3), dtype=torch.float32, device=self.device)
        it = cand = nodes = None
        if stats:
            it = torch.empty(n, dtype=torch.int32, device=self.device)
            cand = torch.empty(n, dtype=torch.int32, device=self.device)
            nodes = torch.empty(n, dtype=torch.int32, device=self.device)
        g = None if guess is None else _dev(guess, torch.float32, self.device).reshape(-1, 3)
        opts = L.DrbNewtonOpts(tol, max_steps, guess_mode, None if g is None else g.data_ptr())
        st = L.DrbQueryStats(None if it is None else it.data_ptr(),
                             None if cand is None else cand.data_ptr(),
                             None if nodes is None else nodes.data_ptr())
        b = self.get_bvh(stream)
        d = self.desc(packed)
        bd = b.desc()
        L.check(L.lib().drb_locate(C.byref(d), C.byref(bd), _ptr(pts), n, C.byref(opts),
                                   _ptr(cell), _ptr(ref), st, _stream(stream)), "drb_locate")
        if stats:
            return cell, ref, it, cand, nodes
        return cell, ref


def _locate_outputs(n, device, stats):
    cell = torch.empty(n, dtype=torch.int32, device=device)
    ref = torch.empty((n, 3), dtype=torch.float32, device=device)
    st = [torch.empty(n, dtype=torch.int32, device=device) for _ in range(3)] if stats else None
    qs = L.DrbQueryStats(*(None if st is None else t.data_ptr() for t in (st or [None] * 3)))
    return cell, ref, st, qs


class BatchedLocator:
    """Persistent, batched Mesh::locate (drb_locate_batched): Morton-ordered
    queries, a global work queue, autotuned launch shape."""

    def __init__(self, mesh: UnstructuredMesh, tol: float = 1e-5, max_steps: int = 20,
                 guess_mode: int = L.GUESS_ELEM_CENTER, config: L.DrbLocateConfig | None = None,
                 bvh: BVH | None = None):
        self.mesh = mesh
        self.tol, self.max_steps, self.guess_mode = tol, max_steps, guess_mode
        self.config = config
        self.bvh = bvh  # None: the mesh's own BVH (with its wide tree)

    def _bvh(self, stream=None) -> BVH:
        b = self.bvh if self.bvh is not None else self.mesh.get_bvh(stream)
        if (self.guess_mode == L.GUESS_SUBBOX_LINEAR and b.leaf_maps is None
                and self.mesh.dim == 3):
            b.build_leaf_maps(self.mesh, stream)
        return b

    def tune(self, sample_points, stream=None):
        pts = _dev(sample_points, torch.float32, self.mesh.device).reshape(-1, 3)
        best = L.DrbLocateConfig()
        ms = C.c_float()
        opts = L.DrbNewtonOpts(self.tol, self.max_steps, self.guess_mode, None)
        bd = self._bvh(stream).desc()  # first: it may add the mesh's hull planes
        d = self.mesh.desc()
        L.check(L.lib().drb_locate_tune(C.byref(d), C.byref(bd), _ptr(pts), pts.shape[0],
                                        C.byref(opts), C.byref(best), C.byref(ms),
                                        _stream(stream)), "drb_locate_tune")
        self.config = best
        return best, ms.value

    def order(self, points, stream=None):
        pts = _dev(points, torch.float32, self.mesh.device).reshape(-1, 3)
        o = torch.empty(pts.shape[0], dtype=torch.int32, device=self.mesh.device)
        bd = self._bvh(stream).desc()
        L.check(L.lib().drb_query_order(C.byref(bd), _ptr(pts), pts.shape[0], _ptr(o),
                                        _stream(stream)), "drb_query_order")
        return o

    def stage(self, points, stream=None):
        """Query records (x, y, z, input index bits) in processing order
        (drb_query_stage), as a float32 tensor of shape (n, 4)."""
        pts = _dev(points, torch.float32, self.mesh.device).reshape(-1, 3)
        rec = torch.empty((pts.shape[0], 4), dtype=torch.float32, device=self.mesh.device)
        bd = self._bvh(stream).desc()
        L.check(L.lib().drb_query_stage(C.byref(bd), _ptr(pts), pts.shape[0], _ptr(rec),
                                        _stream(stream)), "drb_query_stage")
        return rec

    def locate_staged(self, staged, out=None, records=False, stream=None):
        """The persistent kernel alone on staged records (drb_locate_staged).
        records=True: returns (n, 4) records (cell bits, r, s, t) in the
        staged order; else (cell, ref) at the queries' input indices, as
        drb_locate_batched writes them (out = (cell, ref) to reuse)."""
        n = staged.shape[0]
        dev = self.mesh.device
        opts = L.DrbNewtonOpts(self.tol, self.max_steps, self.guess_mode, None)
        cfg = None if self.config is None else C.byref(self.config)
        bd = self._bvh(stream).desc()  # first: it may add the mesh's hull planes
        d = self.mesh.desc()
        if records:
            res = torch.empty((n, 4), dtype=torch.float32, device=dev) if out is None else out
            cell = ref = None
        else:
            res = None
            cell, ref = out if out is not None else (
                torch.empty(n, dtype=torch.int32, device=dev),
                torch.empty((n, 3), dtype=torch.float32, device=dev))
        L.check(L.lib().drb_locate_staged(C.byref(d), C.byref(bd), _ptr(staged), n,
                                          C.byref(opts), cfg, _ptr(res), _ptr(cell), _ptr(ref),
                                          L.DrbQueryStats(), _stream(stream)),
                "drb_locate_staged")
        return res if records else (cell, ref)

    def locate(self, points, order=None, guess=None, stats=False, out=None, stream=None):
        pts = _dev(points, torch.float32, self.mesh.device).reshape(-1, 3)
        n = pts.shape[0]
        if out is None:
            cell, ref, st, qs = _locate_outputs(n, self.mesh.device, stats)
        else:
            cell, ref = out
            st, qs = None, L.DrbQueryStats()
        mode = self.guess_mode if guess is None else L.GUESS_GIVEN
        opts = L.DrbNewtonOpts(self.tol, self.max_steps, mode,
                               None if guess is None else guess.data_ptr())
        cfg = None if self.config is None else C.byref(self.config)
        bd = self._bvh(stream).desc()  # first: it may add the mesh's hull planes
        d = self.mesh.desc()
        if order is None:
            L.check(L.lib().drb_locate_batched(C.byref(d), C.byref(bd), _ptr(pts), n,
                                               C.byref(opts), cfg, _ptr(cell), _ptr(ref), qs,
                                               _stream(stream)), "drb_locate_batched")
        else:
            L.check(L.lib().drb_locate_ordered(C.byref(d), C.byref(bd), _ptr(pts), n,
                                               _ptr(order), C.byref(opts), cfg, _ptr(cell),
                                               _ptr(ref), qs, _stream(stream)),
                    "drb_locate_ordered")
        if stats:
            return cell, ref, st[0], st[1], st[2]
        return cell, ref


    def capture(self, n: int) -> "LocateGraph":
        """A CUDA graph of this locator's batched locate over a static buffer
        of n queries (query order, persistent kernel and their scratch
        allocations), for callers that locate many batches of one size."""
        return LocateGraph(self, n)

    def locate_host(self, host_points, out, chunk: int = 0, stream=None):
        """Locate points held in (page-locked) host memory, writing cell ids
        and reference points into the host tensors out = (cell, ref); the
        copies of consecutive chunks overlap the locate (drb_locate_host)."""
        assert host_points.device.type == "cpu" and host_points.dtype == torch.float32
        cell, ref = out
        assert cell.device.type == "cpu" and ref.device.type == "cpu"
        n = host_points.shape[0]
        opts = L.DrbNewtonOpts(self.tol, self.max_steps, self.guess_mode, None)
        cfg = None if self.config is None else C.byref(self.config)
        bd = self._bvh(stream).desc()  # first: it may add the mesh's hull planes
        d = self.mesh.desc()
        L.check(L.lib().drb_locate_host(C.byref(d), C.byref(bd), _ptr(host_points), n,
                                        C.byref(opts), cfg, chunk, _ptr(cell), _ptr(ref),
                                        _stream(stream)), "drb_locate_host")
        return cell, ref


class LocateGraph:
    """Batched locate of a fixed-size query buffer captured once into a CUDA
    graph and replayed per batch: the queries go into `points` (or are
    passed to run()), results come back in `cell` / `ref`.  The graph holds
    the Morton ordering, the persistent kernel and their stream-ordered
    scratch allocations, so a replay is one launch from the host."""

    def __init__(self, locator: BatchedLocator, n: int):
        dev = locator.mesh.device
        self.locator = locator
        self.points = torch.zeros((n, 3), dtype=torch.float32, device=dev)
        self.cell = torch.empty(n, dtype=torch.int32, device=dev)
        self.ref = torch.empty((n, 3), dtype=torch.float32, device=dev)
        # warm up outside the capture: lazy BVH build and one-time pool setup
        locator.locate(self.points, out=(self.cell, self.ref))
        torch.cuda.synchronize(dev)
        self.graph = torch.cuda.CUDAGraph()
        side = torch.cuda.Stream(dev)
        side.wait_stream(torch.cuda.current_stream(dev))
        with torch.cuda.stream(side):
            locator.locate(self.points, out=(self.cell, self.ref))
        torch.cuda.current_stream(dev).wait_stream(side)
        torch.cuda.synchronize(dev)
        with torch.cuda.graph(self.graph):
            locator.locate(self.points, out=(self.cell, self.ref))

    def run(self, points=None):
        if points is not None:
            self.points.copy_(_dev(points, torch.float32, self.points.device).reshape(-1, 3),
                              non_blocking=True)
        self.graph.replay()
        return self.cell, self.ref


def elem_subboxes(mesh: UnstructuredMesh, stream=None):
    """Per-element sub-boxes (aabbs6, prim_ids, ref_boxes, bounds6) on device."""
    nb = 33 if mesh.dim == 3 else 17
    n = mesh.n_elem * nb
    dev = mesh.device
    aabbs = torch.empty((n, 6), dtype=torch.float32, device=dev)
    prim = torch.empty(n, dtype=torch.int32, device=dev)
    rbf = L.lib().drb_ref_box_floats(mesh.shape, mesh.dim)
    refb = torch.empty((n, rbf), dtype=torch.float32, device=dev)
    bounds = torch.empty(6, dtype=torch.float32, device=dev)
    d = mesh.desc()
    L.check(L.lib().drb_elem_subboxes(C.byref(d), _ptr(aabbs), _ptr(prim), _ptr(refb),
                                      _ptr(bounds), _stream(stream)), "drb_elem_subboxes")
    return aabbs, prim, refb, bounds


def morton_codes(aabbs6: torch.Tensor, bounds6: torch.Tensor, stream=None):
    n = aabbs6.shape[0]
    codes = torch.empty(n, dtype=torch.int32, device=aabbs6.device)
    L.check(L.lib().drb_morton_codes(_ptr(aabbs6), n, _ptr(bounds6), _ptr(codes),
                                     _stream(stream)), "drb_morton_codes")
    return codes


def radix_sort_pairs(keys: torch.Tensor, vals: torch.Tensor, bits: int = 32, stream=None):
    n = keys.numel()
    ko = torch.empty_like(keys)
    vo = torch.empty_like(vals)
    L.check(L.lib().drb_radix_sort_pairs(_ptr(keys), _ptr(vals), _ptr(ko), _ptr(vo), n, bits,
                                         _stream(stream)), "drb_radix_sort_pairs")
    return ko, vo
