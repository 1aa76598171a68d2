// Uniform-grid candidate lists over the leaves of a built BVH.
//
// The batched locate spends about half of its time walking the tree to the
// first candidate leaf (12 wide-node visits of 112 bytes per query on the
// 64^3 mesh).  Because a leaf is a traversal candidate exactly when its own
// box holds the point, and the left-first traversal meets leaves in index
// order, a list per grid cell of the leaves whose boxes overlap the cell,
// sorted by leaf index, yields the same candidates in the same order: the
// point's cell gives a short contiguous run of leaf indices whose boxes
// (a 32-byte record per leaf) are tested instead of a chain of dependent
// node loads.  No reference counterpart (the reference traverses its binary
// nodes, data_model/device_mesh.hpp:262-318).
//
// Build: the leaf boxes are read back out of their parents' node records
// (the same floats the traversal tests), each leaf is filed under every
// cell its box overlaps (grid_axis of its corners), the (cell, leaf) pairs
// are sorted stably by cell (the sorted leaf indices are the entries), the
// per-cell starts are found by binary search, and the box table is written
// once per leaf.
#include "drb_common.cuh"
#include "drb_internal.h"
#include "locate.cuh"

#include <algorithm>
#include <cmath>

namespace drb
{
namespace
{

constexpr long long kMaxCells = 1ll << 28;
constexpr int kMaxDim = 4096;

struct GridGeom
{
  int dims[3];
  float origin[3];
  float inv[3];
};

GridGeom geom_of (const drb_bvh *b)
{
  GridGeom g;
  for (int d = 0; d < 3; ++d)
  {
    g.dims[d] = b->grid_dims[d];
    g.origin[d] = b->grid_origin[d];
    g.inv[d] = b->grid_inv[d];
  }
  return g;
}

// Leaf boxes out of the binary node records (4 x float4 per node: left box
// lo.xyz hi.xyz, right box lo.xyz hi.xyz, child codes; a leaf child is
// -(leaf + 1)).  boxes[6 k ..] = lo.xyz, hi.xyz of sorted leaf k.
__global__ void leaf_boxes_kernel (const float4 *__restrict__ nodes, int n_inner,
                                   float *__restrict__ boxes)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_inner) return;
  const float4 a = __ldg (nodes + 4 * (size_t)i);
  const float4 b = __ldg (nodes + 4 * (size_t)i + 1);
  const float4 c = __ldg (nodes + 4 * (size_t)i + 2);
  const float4 d = __ldg (nodes + 4 * (size_t)i + 3);
  const int l = __float_as_int (d.x), r = __float_as_int (d.y);
  if (l < 0)
  {
    float *o = boxes + 6 * (size_t)(-l - 1);
    o[0] = a.x, o[1] = a.y, o[2] = a.z, o[3] = a.w, o[4] = b.x, o[5] = b.y;
  }
  if (r < 0)
  {
    float *o = boxes + 6 * (size_t)(-r - 1);
    o[0] = b.z, o[1] = b.w, o[2] = c.x, o[3] = c.y, o[4] = c.z, o[5] = c.w;
  }
}

// Sum of the leaf extents per axis (double atomics, one per block and axis).
__global__ void extent_sum_kernel (const float *__restrict__ boxes, int n, double *__restrict__ sum)
{
  double s[3] = { 0.0, 0.0, 0.0 };
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
  {
    const float *b = boxes + 6 * (size_t)k;
    for (int d = 0; d < 3; ++d) s[d] += (double)b[3 + d] - (double)b[d];
  }
  for (int d = 0; d < 3; ++d)
  {
    for (int o = 16; o > 0; o >>= 1) s[d] += __shfl_down_sync (0xffffffffu, s[d], o);
    if ((threadIdx.x & 31) == 0) atomicAdd (sum + d, s[d]);
  }
}

DRB_D void cell_range (const GridGeom &g, const float *b, int (&c0)[3], int (&c1)[3])
{
  for (int d = 0; d < 3; ++d)
  {
    c0[d] = grid_axis (b[d], g.origin[d], g.inv[d], g.dims[d]);
    c1[d] = grid_axis (b[3 + d], g.origin[d], g.inv[d], g.dims[d]);
  }
}

// Cells per leaf, and their sum (64-bit).
__global__ void pair_count_kernel (GridGeom g, const float *__restrict__ boxes, int n,
                                   int *__restrict__ counts, unsigned long long *__restrict__ total)
{
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long c = 0;
  if (k < n)
  {
    int c0[3], c1[3];
    cell_range (g, boxes + 6 * (size_t)k, c0, c1);
    c = (unsigned long long)(c1[0] - c0[0] + 1) * (c1[1] - c0[1] + 1) * (c1[2] - c0[2] + 1);
    if (counts) counts[k] = (int)c;
  }
  for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync (0xffffffffu, c, o);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd (total, c);
}

// (cell, leaf) pairs of every leaf, written from its offset in leaf order.
__global__ void pair_emit_kernel (GridGeom g, const float *__restrict__ boxes, int n,
                                  const int *__restrict__ offsets, unsigned *__restrict__ keys,
                                  int *__restrict__ vals)
{
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  int c0[3], c1[3];
  cell_range (g, boxes + 6 * (size_t)k, c0, c1);
  int o = offsets[k];
  for (int z = c0[2]; z <= c1[2]; ++z)
    for (int y = c0[1]; y <= c1[1]; ++y)
      for (int x = c0[0]; x <= c1[0]; ++x)
      {
        keys[o] = (unsigned)((z * g.dims[1] + y) * g.dims[0] + x);
        vals[o] = k;
        ++o;
      }
}

// Box table: per leaf its box and element (32 bytes, float4 aligned).
__global__ void box_table_kernel (const float *__restrict__ boxes, int n,
                                  const int *__restrict__ leaf_nodes, float4 *__restrict__ table)
{
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const float *b = boxes + 6 * (size_t)k;
  table[2 * (size_t)k] = make_float4 (b[0], b[1], b[2], __int_as_float (__ldg (leaf_nodes + k)));
  table[2 * (size_t)k + 1] = make_float4 (b[3], b[4], b[5], 0.f);
}

// start[c] = first sorted pair whose cell is >= c (lower bound), and
// start[n_cells] = m.
__global__ void cell_start_kernel (const unsigned *__restrict__ keys, int m, long long n_cells,
                                   int *__restrict__ start)
{
  const long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (c > n_cells) return;
  if (c == n_cells)
  {
    start[c] = m;
    return;
  }
  int lo = 0, hi = m;
  while (lo < hi)
  {
    const int mid = (lo + hi) >> 1;
    if ((long long)keys[mid] < c) lo = mid + 1;
    else hi = mid;
  }
  start[c] = lo;
}

int check_bvh (const drb_bvh *b, const char *what)
{
  if (!b || b->n_leaf < 2 || !b->inner_nodes || !b->leaf_nodes)
  {
    set_last_error (what);
    return DRB_ERR_INVALID_ARG;
  }
  return DRB_OK;
}

int leaf_boxes (const drb_bvh *b, float *boxes, cudaStream_t s)
{
  leaf_boxes_kernel<<<div_up (b->n_inner, 256), 256, 0, s>>> ((const float4 *)b->inner_nodes,
                                                              b->n_inner, boxes);
  return check_launch ("leaf_boxes_kernel");
}

} // namespace
} // namespace drb

using namespace drb;

extern "C" int drb_bvh_grid_size (drb_bvh *bvh, float cell_scale, long long *n_entries, void *stream)
{
  if (int st = check_bvh (bvh, "bvh_grid_size: needs a built BVH with at least two leaves")) return st;
  if (!n_entries || !(cell_scale > 0.f) || !std::isfinite (cell_scale))
  {
    set_last_error ("bvh_grid_size: bad arguments");
    return DRB_ERR_INVALID_ARG;
  }
  cudaStream_t s = (cudaStream_t)stream;
  const int n = bvh->n_leaf;
  Scratch scr (s);
  float *boxes = scr.alloc<float> (6 * (size_t)n);
  double *sum = scr.alloc<double> (3);
  unsigned long long *total = scr.alloc<unsigned long long> (1);
  if (!boxes || !sum || !total) return status_from (scr.err);
  if (int st = leaf_boxes (bvh, boxes, s)) return st;
  cudaMemsetAsync (sum, 0, 3 * sizeof (double), s);
  cudaMemsetAsync (total, 0, sizeof (unsigned long long), s);
  extent_sum_kernel<<<std::min (div_up (n, 256), 4 * sm_count ()), 256, 0, s>>> (boxes, n, sum);
  if (int st = check_launch ("extent_sum_kernel")) return st;
  double h_sum[3];
  cudaMemcpyAsync (h_sum, sum, sizeof h_sum, cudaMemcpyDeviceToHost, s);
  if (cudaError_t e = cudaStreamSynchronize (s))
  {
    set_last_error ("bvh_grid_size: extent reduction failed");
    return status_from (e);
  }
  // cells about cell_scale times the mean leaf extent per axis
  double ext[3], want[3];
  for (int d = 0; d < 3; ++d)
  {
    ext[d] = (double)bvh->bounds[2 * d + 1] - (double)bvh->bounds[2 * d];
    const double mean = h_sum[d] / n;
    want[d] = (ext[d] > 0.0 && mean > 0.0) ? std::ceil (ext[d] / (cell_scale * mean)) : 1.0;
    want[d] = std::min (std::max (want[d], 1.0), (double)kMaxDim);
  }
  double cells = want[0] * want[1] * want[2];
  if (cells > (double)kMaxCells)
  {
    const double f = std::cbrt ((double)kMaxCells / cells);
    for (int d = 0; d < 3; ++d) want[d] = std::max (1.0, std::floor (want[d] * f));
  }
  GridGeom g;
  for (int d = 0; d < 3; ++d)
  {
    g.dims[d] = (int)want[d];
    g.origin[d] = bvh->bounds[2 * d];
    g.inv[d] = ext[d] > 0.0 ? (float)(g.dims[d] / ext[d]) : 0.f;
    bvh->grid_dims[d] = g.dims[d];
    bvh->grid_origin[d] = g.origin[d];
    bvh->grid_inv[d] = g.inv[d];
  }
  pair_count_kernel<<<div_up (n, 256), 256, 0, s>>> (g, boxes, n, nullptr, total);
  if (int st = check_launch ("pair_count_kernel")) return st;
  unsigned long long h_total = 0;
  cudaMemcpyAsync (&h_total, total, sizeof h_total, cudaMemcpyDeviceToHost, s);
  if (cudaError_t e = cudaStreamSynchronize (s))
  {
    set_last_error ("bvh_grid_size: pair count failed");
    return status_from (e);
  }
  *n_entries = (long long)h_total;
  return DRB_OK;
}

extern "C" int drb_bvh_grid_build (const drb_bvh *bvh, void *stream)
{
  if (int st = check_bvh (bvh, "bvh_grid_build: needs a built BVH with at least two leaves")) return st;
  if (!bvh->grid_start || !bvh->grid_entries || !bvh->grid_boxes)
  {
    set_last_error ("bvh_grid_build: grid_start, grid_entries and grid_boxes must be set");
    return DRB_ERR_INVALID_ARG;
  }
  const GridGeom g = geom_of (bvh);
  const long long n_cells = (long long)g.dims[0] * g.dims[1] * g.dims[2];
  if (g.dims[0] < 1 || g.dims[1] < 1 || g.dims[2] < 1 || n_cells > kMaxCells)
  {
    set_last_error ("bvh_grid_build: call drb_bvh_grid_size first");
    return DRB_ERR_INVALID_ARG;
  }
  cudaStream_t s = (cudaStream_t)stream;
  const int n = bvh->n_leaf;
  Scratch scr (s);
  float *boxes = scr.alloc<float> (6 * (size_t)n);
  int *counts = scr.alloc<int> (n);
  int *offsets = scr.alloc<int> (n);
  unsigned long long *total = scr.alloc<unsigned long long> (1);
  if (!boxes || !counts || !offsets || !total) return status_from (scr.err);
  if (int st = leaf_boxes (bvh, boxes, s)) return st;
  cudaMemsetAsync (total, 0, sizeof (unsigned long long), s);
  pair_count_kernel<<<div_up (n, 256), 256, 0, s>>> (g, boxes, n, counts, total);
  if (int st = check_launch ("pair_count_kernel")) return st;
  unsigned long long h_total = 0;
  cudaMemcpyAsync (&h_total, total, sizeof h_total, cudaMemcpyDeviceToHost, s);
  if (cudaError_t e = cudaStreamSynchronize (s))
  {
    set_last_error ("bvh_grid_build: pair count failed");
    return status_from (e);
  }
  if (h_total >= (1ull << 31))
  {
    set_last_error ("bvh_grid_build: 2^31 entries or more; use a larger cell_scale");
    return DRB_ERR_UNSUPPORTED;
  }
  const int m = (int)h_total;
  if (int st = exclusive_scan_i32 (counts, offsets, n, nullptr, s)) return st;
  unsigned *keys = scr.alloc<unsigned> (m);
  int *vals = scr.alloc<int> (m);
  unsigned *keys_s = scr.alloc<unsigned> (m);
  if (!keys || !vals || !keys_s) return status_from (scr.err);
  pair_emit_kernel<<<div_up (n, 256), 256, 0, s>>> (g, boxes, n, offsets, keys, vals);
  if (int st = check_launch ("pair_emit_kernel")) return st;
  int bits = 1;
  while ((1ll << bits) < n_cells) ++bits;
  // the sorted leaf indices are the entries
  if (int st = radix_sort_pairs (keys, vals, keys_s, bvh->grid_entries, m, bits, s)) return st;
  box_table_kernel<<<div_up (n, 256), 256, 0, s>>> (boxes, n, bvh->leaf_nodes,
                                                    (float4 *)bvh->grid_boxes);
  if (int st = check_launch ("box_table_kernel")) return st;
  cell_start_kernel<<<div_up (n_cells + 1, 256), 256, 0, s>>> (keys_s, m, n_cells, bvh->grid_start);
  return check_launch ("cell_start_kernel");
}
