"""Test oracle: ctypes wrapper over oracle/libdrb_oracle.so, the CPU
restatement of the reference's point-location algorithm (drb_oracle.cpp).

Test infrastructure only: imported by tests/, __graft_entry__.smoke() and the
bench's CPU-baseline leg, never by the product.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "libdrb_oracle.so"
_lib = None


def available() -> bool:
    return LIB.exists()


def lib():
    global _lib
    if _lib is None:
        if not LIB.exists():
            raise FileNotFoundError(f"{LIB} not built (make -C oracle restate)")
        L = C.CDLL(str(LIB))
        vp = C.c_void_p
        L.orc_hex_eval_d.argtypes = [C.c_int, C.c_int, vp, C.c_int, vp, vp, vp]
        L.orc_locate.argtypes = [C.c_int, C.c_int, vp, vp, C.c_int, vp, vp, vp, vp, C.c_int, vp,
                                 C.c_float, C.c_int, C.c_int, vp, C.c_int, C.c_int, vp, vp, vp,
                                 vp]
        L.orc_newton_fp64.argtypes = [C.c_int, vp, vp, C.c_int, vp, vp, vp, vp]
        L.orc_tet_subboxes.argtypes = [C.c_int, C.c_int, vp, vp, C.c_int, vp, vp]
        L.orc_tet_eval_d.argtypes = [C.c_int, C.c_int, vp, C.c_int, vp, vp, vp]
        L.orc_locate_tet.argtypes = [C.c_int, vp, vp, vp, vp, vp, vp, C.c_int, vp, C.c_float,
                                     C.c_int, C.c_int, vp, C.c_int, C.c_int, vp, vp, vp, vp]
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def hex_eval_d(p: int, cp: np.ndarray, ref: np.ndarray):
    """FP64 value and Jacobian columns of one hex element at reference points."""
    cp = np.ascontiguousarray(cp, np.float64)
    ncomp = cp.size // ((p + 1) ** 3)
    ref = np.ascontiguousarray(ref, np.float64).reshape(-1, 3)
    n = ref.shape[0]
    X = np.zeros((n, ncomp))
    J = np.zeros((n, 3, ncomp))
    lib().orc_hex_eval_d(p, ncomp, _p(cp), n, _p(ref), _p(X), _p(J))
    return X, J


def locate(p, ctrl_idx, xyz, bvh, pts, tol=1e-4, max_steps=20, guess_mode=0, guess=None,
           use_double=False, local_frame=False):
    """Restated DeviceMesh::locate over a BVH given as numpy arrays
    (inner [n_inner,16], leaf_nodes, aabb_ids, ref_boxes [n_leaf,6])."""
    ctrl_idx = np.ascontiguousarray(ctrl_idx, np.int32)
    xyz = np.ascontiguousarray(xyz, np.float32)
    pts = np.ascontiguousarray(pts, np.float32).reshape(-1, 3)
    inner = np.ascontiguousarray(bvh["inner"], np.float32)
    leaf = np.ascontiguousarray(bvh["leaf_nodes"], np.int32)
    ids = np.ascontiguousarray(bvh["aabb_ids"], np.int32)
    refb = np.ascontiguousarray(bvh["ref_boxes"], np.float32)
    g = None if guess is None else np.ascontiguousarray(guess, np.float32)
    n = pts.shape[0]
    cell = np.zeros(n, np.int32)
    ref = np.zeros((n, 3), np.float32)
    it = np.zeros(n, np.int32)
    ca = np.zeros(n, np.int32)
    nd = (p + 1) ** 3
    lib().orc_locate(p, ctrl_idx.size // nd, _p(ctrl_idx), _p(xyz), inner.shape[0], _p(inner),
                     _p(leaf), _p(ids), _p(refb), n, _p(pts), tol, max_steps, guess_mode, _p(g),
                     int(use_double), int(local_frame), _p(cell), _p(ref), _p(it), _p(ca))
    return cell, ref, it, ca


def newton_fp64(p, ctrl_idx, xyz, elem, pts):
    """FP64 solution of each (point, element) pair; (ref [n,3] float64, ok [n])."""
    ctrl_idx = np.ascontiguousarray(ctrl_idx, np.int32)
    xyz = np.ascontiguousarray(xyz, np.float32)
    elem = np.ascontiguousarray(elem, np.int32)
    pts = np.ascontiguousarray(pts, np.float32).reshape(-1, 3)
    n = pts.shape[0]
    out = np.zeros((n, 3))
    ok = np.zeros(n, np.int32)
    lib().orc_newton_fp64(p, _p(ctrl_idx), _p(xyz), n, _p(elem), _p(pts), _p(out), _p(ok))
    return out, ok.astype(bool)


def tet_subboxes(p, ctrl_idx, xyz, reference_index=False):
    """Restated construct_bvh sub-boxes of an order-p tet mesh:
    (aabbs6 [n*33, 6], ref12 [n*33, 12]).  reference_index=True uses the
    reference's own split indexing (cartesian_to_tet_idx)."""
    ctrl_idx = np.ascontiguousarray(ctrl_idx, np.int32)
    xyz = np.ascontiguousarray(xyz, np.float32)
    nd = (p + 1) * (p + 2) * (p + 3) // 6
    n = ctrl_idx.size // nd
    aabbs = np.zeros((n * 33, 6), np.float32)
    refs = np.zeros((n * 33, 12), np.float32)
    lib().orc_tet_subboxes(p, n, _p(ctrl_idx), _p(xyz), int(reference_index), _p(aabbs), _p(refs))
    return aabbs, refs


def tet_eval_d(p: int, cp: np.ndarray, ref: np.ndarray):
    """FP64 value and Jacobian columns of one tet element at reference points."""
    cp = np.ascontiguousarray(cp, np.float64)
    nd = (p + 1) * (p + 2) * (p + 3) // 6
    ncomp = cp.size // nd
    ref = np.ascontiguousarray(ref, np.float64).reshape(-1, 3)
    n = ref.shape[0]
    X = np.zeros((n, ncomp))
    J = np.zeros((n, 3, ncomp))
    lib().orc_tet_eval_d(p, ncomp, _p(cp), n, _p(ref), _p(X), _p(J))
    return X, J


def locate_tet(p, ctrl_idx, xyz, bvh, pts, tol=1e-4, max_steps=20, guess_mode=0, guess=None,
               use_double=False, local_frame=False):
    """Restated DeviceMesh::locate over an order-p tet mesh and a BVH given
    as numpy arrays (ref_boxes [n_leaf, 12])."""
    ctrl_idx = np.ascontiguousarray(ctrl_idx, np.int32)
    xyz = np.ascontiguousarray(xyz, np.float32)
    pts = np.ascontiguousarray(pts, np.float32).reshape(-1, 3)
    inner = np.ascontiguousarray(bvh["inner"], np.float32)
    leaf = np.ascontiguousarray(bvh["leaf_nodes"], np.int32)
    ids = np.ascontiguousarray(bvh["aabb_ids"], np.int32)
    refb = np.ascontiguousarray(bvh["ref_boxes"], np.float32)
    g = None if guess is None else np.ascontiguousarray(guess, np.float32)
    n = pts.shape[0]
    cell = np.zeros(n, np.int32)
    ref = np.zeros((n, 3), np.float32)
    it = np.zeros(n, np.int32)
    ca = np.zeros(n, np.int32)
    lib().orc_locate_tet(p, _p(ctrl_idx), _p(xyz), _p(inner), _p(leaf), _p(ids), _p(refb), n,
                         _p(pts), tol, max_steps, guess_mode, _p(g), int(use_double),
                         int(local_frame), _p(cell), _p(ref), _p(it), _p(ca))
    return cell, ref, it, ca
