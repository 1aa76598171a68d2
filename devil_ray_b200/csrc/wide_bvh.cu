// 4-wide collapse of the reference-layout binary LBVH, for traversal only.
//
// Every binary inner node at even depth becomes one 128-byte wide node whose
// (up to) four children are its grandchildren, or its children where those
// are leaves, in left-to-right order.  A query then makes one dependent
// 128-byte load per two binary levels.  The child boxes are copied bit for
// bit from the binary records, and a parent box is the exact union of its
// children's, so a leaf is reached in the wide tree exactly when its own box
// holds the point, as in the binary tree (linear_bvh_builder.cpp:253-397,
// device_mesh.hpp:262-318); visiting the hit children lowest first keeps
// the binary traversal's left-first leaf order.  Point location over the
// wide tree therefore tries the same candidates in the same order and
// returns the same result.
//
//   parent_kernel    parent index of every binary inner node
//   depth_kernel     depth by walking the parents (bounded), even -> wide
//   (exclusive scan of the flags gives each wide node its index)
//   wide_emit_kernel one thread per wide node gathers its children
#include "drb_common.cuh"
#include "drb_internal.h"
#include "locate.cuh"

namespace drb
{
namespace
{

constexpr int kMaxWalk = 1024; // depth bound of the parent walk

__global__ void parent_kernel (const float4 *__restrict__ nodes, int n_inner, int *__restrict__ parent)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_inner) return;
  if (i == 0) parent[0] = -1;
  const float4 d = nodes[4 * (size_t)i + 3];
  const int l = __float_as_int (d.x), r = __float_as_int (d.y);
  if (l >= 0 && l / 4 < n_inner) parent[l / 4] = i;
  if (r >= 0 && r / 4 < n_inner) parent[r / 4] = i;
}

__global__ void depth_kernel (const int *__restrict__ parent, int n_inner, int *__restrict__ wide_flag,
                              int *__restrict__ max_depth)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_inner) return;
  int d = 0, j = i;
  while (d < kMaxWalk)
  {
    const int p = parent[j];
    if (p < 0) break;
    j = p;
    ++d;
  }
  wide_flag[i] = (d & 1) == 0 ? 1 : 0;
  atomicMax (max_depth, d);
}

// box c (0 left, 1 right) of a binary record: lo xyz, hi xyz
DRB_D void record_box (const float4 *__restrict__ rec, int c, float (&b)[6])
{
  const float4 a = rec[0], bb = rec[1], cc = rec[2];
  if (c == 0)
  {
    b[0] = a.x; b[1] = a.y; b[2] = a.z; b[3] = a.w; b[4] = bb.x; b[5] = bb.y;
  }
  else
  {
    b[0] = bb.z; b[1] = bb.w; b[2] = cc.x; b[3] = cc.y; b[4] = cc.z; b[5] = cc.w;
  }
}

__global__ void wide_emit_kernel (const float4 *__restrict__ nodes, int n_inner,
                                  const int *__restrict__ wide_flag, const int *__restrict__ wide_id,
                                  float4 *__restrict__ wide)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_inner || !wide_flag[i]) return;
  float box[4][6];
  int kid[4];
  int k = 0;
  const float4 *rec = nodes + 4 * (size_t)i;
  const float4 d = rec[3];
  const int ch[2] = { __float_as_int (d.x), __float_as_int (d.y) };
#pragma unroll
  for (int c = 0; c < 2; ++c)
  {
    if (ch[c] < 0)
    {
      record_box (rec, c, box[k]);
      kid[k++] = ch[c];
    }
    else
    {
      const float4 *rj = nodes + ch[c];
      const float4 dj = rj[3];
      const int gc[2] = { __float_as_int (dj.x), __float_as_int (dj.y) };
#pragma unroll
      for (int g = 0; g < 2; ++g)
      {
        record_box (rj, g, box[k]);
        kid[k++] = gc[g] < 0 ? gc[g] : wide_id[gc[g] / 4];
      }
    }
  }
  for (int q = k; q < 4; ++q)
  {
    box[q][0] = box[q][1] = box[q][2] = INFINITY;
    box[q][3] = box[q][4] = box[q][5] = -INFINITY;
    kid[q] = kWideEmpty;
  }
  float4 *o = wide + 8 * (size_t)wide_id[i];
#pragma unroll
  for (int f = 0; f < 6; ++f) o[f] = make_float4 (box[0][f], box[1][f], box[2][f], box[3][f]);
  o[6] = make_float4 (__int_as_float (kid[0]), __int_as_float (kid[1]), __int_as_float (kid[2]),
                      __int_as_float (kid[3]));
  o[7] = make_float4 (__int_as_float (k), 0.f, 0.f, 0.f);
}

} // namespace
} // namespace drb

using namespace drb;

extern "C" int drb_bvh_widen (drb_bvh *bvh, float *wide_nodes, int capacity, void *stream)
{
  if (!bvh || !bvh->inner_nodes || bvh->n_inner < 1 || (wide_nodes && capacity < 1))
  {
    set_last_error ("bvh_widen: needs a built BVH");
    return DRB_ERR_INVALID_ARG;
  }
  cudaStream_t s = (cudaStream_t)stream;
  const int n = bvh->n_inner;
  Scratch scr (s);
  int *parent = scr.alloc<int> (n);
  int *flag = scr.alloc<int> (n);
  int *wid = scr.alloc<int> (n);
  int *stat = scr.alloc<int> (2); // [0] max depth, [1] wide count
  if (!stat) return status_from (scr.err);
  cudaMemsetAsync (stat, 0, 2 * sizeof (int), s);
  const float4 *nodes = (const float4 *)bvh->inner_nodes;
  parent_kernel<<<div_up (n, 256), 256, 0, s>>> (nodes, n, parent);
  int st = check_launch ("parent_kernel");
  if (st) return st;
  depth_kernel<<<div_up (n, 256), 256, 0, s>>> (parent, n, flag, stat);
  if ((st = check_launch ("depth_kernel"))) return st;
  if ((st = exclusive_scan_i32 (flag, wid, n, stat + 1, s))) return st;
  int h[2] = { 0, 0 };
  cudaError_t e = cudaMemcpyAsync (h, stat, sizeof (h), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize (s);
  if (e != cudaSuccess)
  {
    set_last_error (cudaGetErrorString (e));
    return status_from (e);
  }
  const int depth = h[0], count = h[1];
  bvh->n_wide = count;
  bvh->wide_depth = depth / 2 + 1;
  if (depth >= kMaxWalk || 3 * bvh->wide_depth + 1 > kWideStack)
  {
    set_last_error ("bvh_widen: tree too deep for the wide traversal stack");
    bvh->wide_nodes = nullptr;
    return DRB_ERR_UNSUPPORTED;
  }
  if (!wide_nodes) return DRB_OK; // size query
  if (capacity < count)
  {
    set_last_error ("bvh_widen: wide node array too small (query the count first)");
    return DRB_ERR_INVALID_ARG;
  }
  wide_emit_kernel<<<div_up (n, 256), 256, 0, s>>> (nodes, n, flag, wid, (float4 *)wide_nodes);
  if ((st = check_launch ("wide_emit_kernel"))) return st;
  bvh->wide_nodes = wide_nodes;
  return DRB_OK;
}
