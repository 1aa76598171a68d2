"""The allocation-free batched locate, called through the C-ABI.

It exists for callers that cannot allocate device memory while they locate
points: a host application whose device memory belongs to its own pool or
allocator, or a latency-critical path that cannot absorb cudaMalloc's
implicit synchronisation.  Its answers must equal those of the allocating
drb_locate_batched on the same inputs, bit for bit, on consecutive calls that
reuse the library's fixed scratch array, and a call must leave the device's
stream-ordered pool and torch's allocator untouched.  This file is collected
last so a failure here cannot hide the result of another test.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _call(lib, L, fn, mesh_d, bvh_d, pts, opts, cell, ref, stream):
    args = [C.byref(mesh_d), C.byref(bvh_d), C.c_void_p(pts.data_ptr()), pts.shape[0],
            C.byref(opts), None, C.c_void_p(cell.data_ptr()), C.c_void_p(ref.data_ptr()),
            L.DrbQueryStats(), C.c_void_p(stream)]
    return getattr(lib, fn)(*args)


def _pool_used_high(device_index):
    """(used bytes now, high-water mark) of the device's default
    stream-ordered pool, where the allocating entry points take scratch."""
    from cuda.bindings import runtime as rt
    err, pool = rt.cudaDeviceGetDefaultMemPool(device_index)
    assert err == rt.cudaError_t.cudaSuccess
    out = []
    for attr in (rt.cudaMemPoolAttr.cudaMemPoolAttrUsedMemCurrent,
                 rt.cudaMemPoolAttr.cudaMemPoolAttrUsedMemHigh):
        err, v = rt.cudaMemPoolGetAttribute(pool, attr)
        assert err == rt.cudaError_t.cudaSuccess
        out.append(int(v))
    return out


def _reset_pool_high(device_index):
    from cuda.bindings import driver
    from cuda.bindings import runtime as rt
    err, pool = rt.cudaDeviceGetDefaultMemPool(device_index)
    assert err == rt.cudaError_t.cudaSuccess
    (err,) = rt.cudaMemPoolSetAttribute(pool, rt.cudaMemPoolAttr.cudaMemPoolAttrUsedMemHigh,
                                        driver.cuuint64_t(0))
    assert err == rt.cudaError_t.cudaSuccess


def test_noalloc_matches_allocating_path_twice(cuda):
    import torch
    from devil_ray_b200 import _lib as L
    from devil_ray_b200 import api, meshgen
    lib = L.lib()
    m = meshgen.trilinear_distorted_mesh(16, 2, 0.15, seed=21)
    mesh = api.UnstructuredMesh(m.ctrl_idx, m.xyz, m.order, device=cuda)
    bvh = mesh.get_bvh()
    mesh_d, bvh_d = mesh.desc(), bvh.desc()
    stream = torch.cuda.current_stream().cuda_stream
    opts = L.DrbNewtonOpts(1e-5, 20, L.GUESS_ELEM_CENTER, None)
    cap = lib.drb_noalloc_max_queries()
    assert cap == 1 << 20
    for call, (count, seed) in enumerate([(300_000, 5), (cap, 6)]):
        pts = torch.as_tensor(meshgen.uniform_queries(count, seed), device=cuda)
        c0 = torch.empty(count, dtype=torch.int32, device=cuda)
        r0 = torch.empty((count, 3), dtype=torch.float32, device=cuda)
        c1 = torch.full_like(c0, -7)
        r1 = torch.full_like(r0, 7.0)
        assert _call(lib, L, "drb_locate_batched", mesh_d, bvh_d, pts, opts, c0, r0, stream) == 0
        torch.cuda.synchronize()
        # the allocating call has returned its scratch; the allocation-free
        # call must take none from the pool nor from torch's allocator
        _reset_pool_high(cuda.index or 0)
        used0, _ = _pool_used_high(cuda.index or 0)
        torch_used0 = torch.cuda.memory_allocated(cuda)
        assert _call(lib, L, "drb_locate_batched_noalloc", mesh_d, bvh_d, pts, opts, c1, r1,
                     stream) == 0, lib.drb_last_error()
        torch.cuda.synchronize()
        used1, high1 = _pool_used_high(cuda.index or 0)
        assert used1 == used0 and high1 <= used0, \
            f"call {call}: pool use moved {used0} -> {used1} (high {high1})"
        assert torch.cuda.memory_allocated(cuda) == torch_used0
        # every query's answer is independent of the processing order, so the
        # two paths agree bit for bit
        assert torch.equal(c0, c1), f"call {call}: cell ids differ"
        assert torch.equal(r0.view(torch.int32), r1.view(torch.int32)), \
            f"call {call}: ref points differ"
        assert 0.85 < (c1 >= 0).float().mean().item() < 0.95


@pytest.mark.parametrize("kind", ["tet", "quad"])
def test_noalloc_other_element_types(cuda, kind):
    """Tet and 2D quad meshes through the allocation-free entry point give
    the allocating path's results."""
    import torch
    from devil_ray_b200 import _lib as L
    from devil_ray_b200 import api, meshgen
    lib = L.lib()
    if kind == "tet":
        m = meshgen.tet_warped_mesh(8, 2, 0.05, jitter=0.01, seed=4)
        mesh = api.UnstructuredMesh(m.ctrl_idx, m.xyz, m.order, device=cuda, shape=L.SHAPE_SIMPLEX)
        pts = torch.as_tensor(meshgen.uniform_queries(200_000, 8), device=cuda)
    else:
        m = meshgen.quad_warped_mesh(24, 2, 0.04, jitter=0.004, seed=4)
        mesh = api.UnstructuredMesh(m.ctrl_idx, m.xyz, m.order, dim=2, device=cuda)
        rng = np.random.default_rng(8)
        xy = rng.uniform(-0.05, 1.05, size=(200_000, 2))
        pts = torch.as_tensor(np.concatenate([xy, np.zeros((200_000, 1))], 1).astype(np.float32),
                              device=cuda)
    bvh = mesh.get_bvh()
    mesh_d, bvh_d = mesh.desc(), bvh.desc()
    stream = torch.cuda.current_stream().cuda_stream
    opts = L.DrbNewtonOpts(1e-5, 20, L.GUESS_ELEM_CENTER, None)
    n = pts.shape[0]
    c0 = torch.empty(n, dtype=torch.int32, device=cuda)
    r0 = torch.empty((n, 3), dtype=torch.float32, device=cuda)
    c1 = torch.full_like(c0, -7)
    r1 = torch.full_like(r0, 7.0)
    assert _call(lib, L, "drb_locate_batched", mesh_d, bvh_d, pts, opts, c0, r0, stream) == 0
    assert _call(lib, L, "drb_locate_batched_noalloc", mesh_d, bvh_d, pts, opts, c1, r1,
                 stream) == 0, lib.drb_last_error()
    torch.cuda.synchronize()
    assert torch.equal(c0, c1)
    assert torch.equal(r0.view(torch.int32), r1.view(torch.int32))
    assert (c1 >= 0).float().mean().item() > 0.8


def test_noalloc_rejects_oversized_call(cuda):
    import torch
    from devil_ray_b200 import _lib as L
    from devil_ray_b200 import api, meshgen
    lib = L.lib()
    m = meshgen.workload_mesh("volume_8")
    mesh = api.UnstructuredMesh(m.ctrl_idx, m.xyz, m.order, device=cuda)
    bvh = mesh.get_bvh()
    opts = L.DrbNewtonOpts(1e-5, 20, L.GUESS_ELEM_CENTER, None)
    n = lib.drb_noalloc_max_queries() + 1
    pts = torch.zeros((n, 3), dtype=torch.float32, device=cuda)
    cell = torch.empty(n, dtype=torch.int32, device=cuda)
    ref = torch.empty((n, 3), dtype=torch.float32, device=cuda)
    st = _call(lib, L, "drb_locate_batched_noalloc", mesh.desc(), bvh.desc(), pts, opts, cell,
               ref, torch.cuda.current_stream().cuda_stream)
    assert st == L.DRB_ERR_INVALID_ARG
    assert b"fixed scratch capacity" in lib.drb_last_error()
