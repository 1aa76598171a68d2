// LBVH construction over Bernstein element sub-boxes, B200-native.
//
// Pipeline (one stream, no host round trip until the final bounds copy):
//   subbox_kernel   warp per element, 32/16 de Casteljau splits held in shared
//                   memory (the reference spills them to a num_els*33*nd
//                   global scratch, data_model/mesh_utils.cpp:552-569), hull
//                   AABBs, x1.000001 scale, block-reduced scene bounds
//   morton_kernel   30-bit codes of the scaled-box centroids
//   radix sort      stable 4-pass LSD sort of (code, sub-box id)  (sort.cu)
//   gather_kernel   sorted AABBs, leaf element ids
//   karras_kernel   Karras 2012 radix tree, index tie-break
//   refit_kernel    bottom-up AABB union with arrival counters
//   emit_kernel     4 x float4 node records
//
// Bit-exactness: the sub-box, scale, measure and Morton arithmetic use
// explicitly rounded intrinsics (__fadd_rn/__fmul_rn/__fsub_rn) in the same
// operation order as the reference so that no FMA contraction changes a
// bit; min/max and the integer tree steps are exact by construction.
#include "bernstein.cuh"
#include "drb_common.cuh"
#include "drb_internal.h"
#include "simplex.cuh"

#include <cstdio>
#include <cstring>
#include <vector>

namespace drb
{

namespace
{

constexpr int kSubboxWarps = 4;

template <int DIM> struct SplitCount
{
  // construct_bvh: splits = 2 * (2 << dim)  (mesh_utils.cpp:527)
  static constexpr int splits = 2 * (2 << DIM);
  static constexpr int boxes = splits + 1;
};

DRB_D float warp_min (float v)
{
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fminf (v, __shfl_xor_sync (0xffffffffu, v, o));
  return v;
}
DRB_D float warp_max (float v)
{
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmaxf (v, __shfl_xor_sync (0xffffffffu, v, o));
  return v;
}

// Hull of nd control points held in shared memory (Element::get_bounds via
// positive_get_bounds, data_model/element.hpp:150-160).
template <int ND>
DRB_D void warp_hull (const float *cps, float *box6, int lane)
{
  float mn[3] = { INFINITY, INFINITY, INFINITY };
  float mx[3] = { -INFINITY, -INFINITY, -INFINITY };
  for (int i = lane; i < ND; i += kWarp)
  {
#pragma unroll
    for (int k = 0; k < 3; ++k)
    {
      const float q = cps[3 * i + k];
      mn[k] = fminf (mn[k], q);
      mx[k] = fmaxf (mx[k], q);
    }
  }
#pragma unroll
  for (int k = 0; k < 3; ++k)
  {
    mn[k] = warp_min (mn[k]);
    mx[k] = warp_max (mx[k]);
  }
  if (lane == 0)
  {
#pragma unroll
    for (int k = 0; k < 3; ++k)
    {
      box6[2 * k] = mn[k];
      box6[2 * k + 1] = mx[k];
    }
  }
}

// AABB::volume, falling back to AABB::surface_area when the volume is 0
// (aabb.hpp:173-195, mesh_utils.cpp:587-603).  Explicit rounding, same order.
DRB_D float box_measure (const float *b)
{
  const float l0 = __fsub_rn (b[1], b[0]);
  const float l1 = __fsub_rn (b[3], b[2]);
  const float l2 = __fsub_rn (b[5], b[4]);
  float vol = __fmul_rn (__fmul_rn (__fmul_rn (1.f, l0), l1), l2);
  if (vol == 0.f)
  {
    float area = __fmul_rn (__fmul_rn (2.f, l0), l1);
    area = __fadd_rn (area, __fmul_rn (__fmul_rn (2.f, l1), l2));
    area = __fadd_rn (area, __fmul_rn (__fmul_rn (2.f, l2), l0));
    vol = area;
  }
  return vol;
}

// Range::scale about the centre (range.hpp:162-172) with the float value of
// the double constant 1.000001 (mesh_utils.cpp:517, aabb.hpp:105-111).
DRB_D void scale_range (float &mn, float &mx, float s)
{
  if (mn > mx) return;
  const float c = __fmul_rn (0.5f, __fadd_rn (mn, mx));
  const float delta = __fmul_rn (__fmul_rn (s, 0.5f), __fsub_rn (mx, mn));
  mn = fminf (mn, __fsub_rn (c, delta));
  mx = fmaxf (mx, __fadd_rn (c, delta));
}

// One half of a binary de Casteljau split at 0.5 along `axis`, in place, for
// `lines x 3` work items spread over the warp (split_inplace<Tensor>,
// data_model/elem_ops.hpp:1346-1405).  left: keep [0,0.5]; else [0.5,1].
template <int DIM, int P>
DRB_D void split_half (float *cps, int axis, bool left, int item)
{
  constexpr int NL = (DIM == 3) ? (P + 1) * (P + 1) : (P + 1);
  const int line = item / 3;
  const int k = item - 3 * line;
  if (line >= NL) return;
  int stride = 1;
  for (int d = 0; d < axis; ++d) stride *= (P + 1);
  const int chunk_sz = stride * (P + 1);
  const int chunk = line / stride;
  const int e = line - chunk * stride;
  const int base = chunk * chunk_sz + e;
  float d[P + 1];
#pragma unroll
  for (int ii = 0; ii <= P; ++ii) d[ii] = cps[3 * (base + ii * stride) + k];
  if (left)
  {
#pragma unroll
    for (int ff = 1; ff <= P; ++ff)
#pragma unroll
      for (int ii = P; ii >= ff; --ii)
        d[ii] = __fadd_rn (__fmul_rn (d[ii - 1], 0.5f), __fmul_rn (d[ii], 0.5f));
  }
  else
  {
#pragma unroll
    for (int fb = 1; fb <= P; ++fb)
#pragma unroll
      for (int ii = 0; ii <= P - fb; ++ii)
        d[ii] = __fadd_rn (__fmul_rn (d[ii], 0.5f), __fmul_rn (d[ii + 1], 0.5f));
  }
#pragma unroll
  for (int ii = 0; ii <= P; ++ii) cps[3 * (base + ii * stride) + k] = d[ii];
}

// Scene bounds (reduce, linear_bvh_builder.cpp:19-58) of the boxes a block
// wrote: warp, then block, then ordered-integer atomics into bounds_ord.
DRB_D void reduce_scene_bounds (float (&bmn)[3], float (&bmx)[3], float (*s_bounds)[6], int warp,
                                int lane, unsigned *bounds_ord)
{
#pragma unroll
  for (int k = 0; k < 3; ++k)
  {
    bmn[k] = warp_min (bmn[k]);
    bmx[k] = warp_max (bmx[k]);
  }
  if (lane == 0)
  {
#pragma unroll
    for (int k = 0; k < 3; ++k)
    {
      s_bounds[warp][2 * k] = bmn[k];
      s_bounds[warp][2 * k + 1] = bmx[k];
    }
  }
  __syncthreads ();
  if (threadIdx.x < 6)
  {
    const int q = threadIdx.x;
    float v = s_bounds[0][q];
    for (int w = 1; w < kSubboxWarps; ++w)
      v = (q & 1) ? fmaxf (v, s_bounds[w][q]) : fminf (v, s_bounds[w][q]);
    if (!isinf (v))
    {
      if (q & 1) atomicMax (bounds_ord + q, float_to_ordered (v));
      else atomicMin (bounds_ord + q, float_to_ordered (v));
    }
  }
}

template <int DIM, int P>
__global__ void __launch_bounds__ (kSubboxWarps * kWarp)
subbox_kernel (const int *__restrict__ ctrl_idx, const float *__restrict__ xyz, int n_elem,
               float *__restrict__ aabbs6, int *__restrict__ prim_ids, float *__restrict__ ref_out,
               unsigned *__restrict__ bounds_ord)
{
  constexpr int ND = (DIM == 3) ? (P + 1) * (P + 1) * (P + 1) : (P + 1) * (P + 1);
  constexpr int NB = SplitCount<DIM>::boxes;
  constexpr int NL = (DIM == 3) ? (P + 1) * (P + 1) : (P + 1);
  constexpr int CPW = NB * ND * 3;     // control point floats per warp
  extern __shared__ float smem[];
  __shared__ float s_bounds[kSubboxWarps][6];

  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  float *cps = smem + warp * CPW;
  float *boxes = smem + kSubboxWarps * CPW + warp * NB * 6;
  float *refs = smem + kSubboxWarps * (CPW + NB * 6) + warp * NB * 2 * DIM;

  const int el = blockIdx.x * kSubboxWarps + warp;
  float bmn[3] = { INFINITY, INFINITY, INFINITY };
  float bmx[3] = { -INFINITY, -INFINITY, -INFINITY };

  if (el < n_elem)
  {
    // box 0: the element itself, ref universe [0,1]^dim
    for (int t = lane; t < ND * 3; t += kWarp)
    {
      const int i = t / 3;
      const int k = t - 3 * i;
      cps[t] = __ldg (xyz + 3 * (size_t)__ldg (ctrl_idx + (size_t)el * ND + i) + k);
    }
    if (lane < DIM)
    {
      refs[lane] = 0.f;
      refs[DIM + lane] = 1.f;
    }
    __syncwarp ();
    warp_hull<ND> (cps, boxes, lane);
    __syncwarp ();

    for (int count = 1; count < NB; ++count)
    {
      // largest-measure box, first one on ties (mesh_utils.cpp:586-603)
      int max_id = 0;
      float max_measure = box_measure (boxes);
      for (int b = 1; b < count; ++b)
      {
        const float m = box_measure (boxes + 6 * b);
        if (m > max_measure)
        {
          max_id = b;
          max_measure = m;
        }
      }
      // pick_binary_split: longest reference axis, first on ties
      // (mesh_utils.cpp:482-506)
      const float *rm = refs + max_id * 2 * DIM;
      int axis = 0;
      float max_len = rm[DIM] - rm[0];
#pragma unroll
      for (int d = 1; d < DIM; ++d)
      {
        const float len = rm[DIM + d] - rm[d];
        if (len > max_len)
        {
          axis = d;
          max_len = len;
        }
      }
      __syncwarp ();
      if (lane == 0)
      {
        // split_subref<Tensor> (data_model/ref_space.hpp:148-171)
        float *rd = refs + count * 2 * DIM;
        float *rmw = refs + max_id * 2 * DIM;
        const float sp = __fadd_rn (__fmul_rn (rmw[axis], 0.5f), __fmul_rn (rmw[DIM + axis], 0.5f));
#pragma unroll
        for (int q = 0; q < 2 * DIM; ++q) rd[q] = rmw[q];
        rmw[DIM + axis] = sp;
        rd[axis] = sp;
      }
      float *mother = cps + max_id * ND * 3;
      float *dghter = cps + count * ND * 3;
      for (int t = lane; t < ND * 3; t += kWarp) dghter[t] = mother[t];
      __syncwarp ();
      for (int item = lane; item < 2 * NL * 3; item += kWarp)
      {
        const bool is_mother = item < NL * 3;
        split_half<DIM, P> (is_mother ? mother : dghter, axis, is_mother,
                            is_mother ? item : item - NL * 3);
      }
      __syncwarp ();
      warp_hull<ND> (mother, boxes + 6 * max_id, lane);
      warp_hull<ND> (dghter, boxes + 6 * count, lane);
      __syncwarp ();
    }

    const float s = (float)1.000001;
    for (int b = lane; b < NB; b += kWarp)
    {
      float bx[6];
#pragma unroll
      for (int q = 0; q < 6; ++q) bx[q] = boxes[6 * b + q];
#pragma unroll
      for (int k = 0; k < 3; ++k) scale_range (bx[2 * k], bx[2 * k + 1], s);
      const size_t o = (size_t)el * NB + b;
#pragma unroll
      for (int q = 0; q < 6; ++q) aabbs6[6 * o + q] = bx[q];
      prim_ids[o] = el;
#pragma unroll
      for (int q = 0; q < 2 * DIM; ++q) ref_out[2 * DIM * o + q] = refs[2 * DIM * b + q];
#pragma unroll
      for (int k = 0; k < 3; ++k)
      {
        bmn[k] = fminf (bmn[k], bx[2 * k]);
        bmx[k] = fmaxf (bmx[k], bx[2 * k + 1]);
      }
    }
  }
  reduce_scene_bounds (bmn, bmx, s_bounds, warp, lane, bounds_ord);
}

// ---- simplex (tet) sub-boxes -------------------------------------------
//
// Same forall as the tensor case (mesh_utils.cpp:557-670, 33 boxes per tet)
// with the simplex split: the reference sub-simplex is four vertices (u, v,
// w axis vertices, then the origin; ref_space.hpp:36-46); the split halves
// its longest edge (first pair v1 < v2 on ties, mesh_utils.cpp:455-480) and
// moves the `displaced` vertex to the midpoint (split_subref<Simplex>,
// ref_space.hpp:133-146); the control points of both halves come from
// de Casteljau along that edge (split_inplace<3,Simplex>,
// elem_ops.hpp:1270-1311).  The reference linearises the dof multi-index
// there with cartesian_to_tet_idx (elem_ops.hpp:32-47), whose in-layer term
// uses the full edge length instead of the layer's: for orders >= 2 it
// addresses the wrong dofs (e.g. order 2 maps (0,1,1) and (0,0,2) both to
// 9) and order 3 reaches index 20 of a 20-dof element.  The layout every
// evaluator uses (the general-order eval_d walk, elem_ops.hpp:945-1030) is
// the layered one of tet_index, which this kernel uses, so its sub-boxes
// bound the split geometry at every order; at order 1 the two indexings
// coincide and the boxes are bit-identical to the reference's.

constexpr int kTetRefFloats = 12; // SubRef<3,Simplex>: four vertices

// One line of a tet split: the dofs with fixed exponents g, h of the two
// vertices off the split edge, ordered by the exponent a of the displaced
// vertex v0 (the tradeoff vertex v1 gets m - a).  De Casteljau at 0.5 in the
// reference's update order: for nu = m..1, a = m down to m - nu + 1,
//   C[a] = C[a] * f + C[a - 1] * (1 - f).
template <int P>
DRB_D void tet_split_line (float *cps, int v0, int v1, int g, int h, int comp)
{
  const int avail = 0xf & ~(1 << v0) & ~(1 << v1);
  const int v2 = (avail & 1) ? 0 : (avail & 2) ? 1 : (avail & 4) ? 2 : 3;
  const int v3 = 6 - v0 - v1 - v2;
  const int m = P - g - h;
  int ids[P + 1];
  float d[P + 1];
#pragma unroll
  for (int a = 0; a <= P; ++a)
  {
    if (a > m) break;
    int b[4];
    b[v0] = a;
    b[v1] = m - a;
    b[v2] = g;
    b[v3] = h;
    ids[a] = tet_index (b[0], b[1], b[2], P);
    d[a] = cps[3 * ids[a] + comp];
  }
#pragma unroll
  for (int nu = P; nu >= 1; --nu)
  {
    if (nu > m) continue;
#pragma unroll
    for (int a = P; a >= 1; --a)
    {
      if (a > m || a < m - nu + 1) continue;
      d[a] = __fadd_rn (__fmul_rn (d[a], 0.5f), __fmul_rn (d[a - 1], 0.5f));
    }
  }
#pragma unroll
  for (int a = 0; a <= P; ++a)
  {
    if (a > m) break;
    cps[3 * ids[a] + comp] = d[a];
  }
}

template <int P>
__global__ void __launch_bounds__ (kSubboxWarps * kWarp)
tet_subbox_kernel (const int *__restrict__ ctrl_idx, const float *__restrict__ xyz, int n_elem,
                   float *__restrict__ aabbs6, int *__restrict__ prim_ids,
                   float *__restrict__ ref_out, unsigned *__restrict__ bounds_ord)
{
  constexpr int ND = tet_dofs<P> ();
  constexpr int NB = SplitCount<3>::boxes;
  constexpr int NL = P * (P + 1) / 2; // lines per split: g + h < P
  constexpr int CPW = NB * ND * 3;
  extern __shared__ float smem[];
  __shared__ float s_bounds[kSubboxWarps][6];

  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  float *cps = smem + warp * CPW;
  float *boxes = smem + kSubboxWarps * CPW + warp * NB * 6;
  float *refs = smem + kSubboxWarps * (CPW + NB * 6) + warp * NB * kTetRefFloats;

  const int el = blockIdx.x * kSubboxWarps + warp;
  float bmn[3] = { INFINITY, INFINITY, INFINITY };
  float bmx[3] = { -INFINITY, -INFINITY, -INFINITY };

  if (el < n_elem)
  {
    for (int t = lane; t < ND * 3; t += kWarp)
    {
      const int i = t / 3;
      const int k = t - 3 * i;
      cps[t] = __ldg (xyz + 3 * (size_t)__ldg (ctrl_idx + (size_t)el * ND + i) + k);
    }
    // ref_universe<Simplex>: unit axis vertices, then the origin
    if (lane < kTetRefFloats) refs[lane] = (lane < 9 && lane % 4 == 0) ? 1.f : 0.f;
    __syncwarp ();
    warp_hull<ND> (cps, boxes, lane);
    __syncwarp ();

    for (int count = 1; count < NB; ++count)
    {
      int max_id = 0;
      float max_measure = box_measure (boxes);
      for (int b = 1; b < count; ++b)
      {
        const float mm = box_measure (boxes + 6 * b);
        if (mm > max_measure)
        {
          max_id = b;
          max_measure = mm;
        }
      }
      // pick_binary_split<Simplex>: longest reference edge (squared length
      // summed in component order), first pair on ties
      const float *rm = refs + max_id * kTetRefFloats;
      int dv = 0, tv = 1;
      float max_l2 = 0.f;
      for (int a = 0; a < 3; ++a)
        for (int b = a + 1; b < 4; ++b)
        {
          const float e0 = __fsub_rn (rm[3 * a], rm[3 * b]);
          const float e1 = __fsub_rn (rm[3 * a + 1], rm[3 * b + 1]);
          const float e2 = __fsub_rn (rm[3 * a + 2], rm[3 * b + 2]);
          const float l2 = __fadd_rn (__fadd_rn (__fmul_rn (e0, e0), __fmul_rn (e1, e1)), __fmul_rn (e2, e2));
          if (l2 > max_l2)
          {
            dv = a;
            tv = b;
            max_l2 = l2;
          }
        }
      __syncwarp ();
      if (lane == 0)
      {
        float *rmw = refs + max_id * kTetRefFloats;
        float *rd = refs + count * kTetRefFloats;
        float sp[3];
#pragma unroll
        for (int k = 0; k < 3; ++k)
          sp[k] = __fadd_rn (__fmul_rn (rmw[3 * tv + k], 0.5f), __fmul_rn (rmw[3 * dv + k], 0.5f));
#pragma unroll
        for (int q = 0; q < kTetRefFloats; ++q) rd[q] = rmw[q];
#pragma unroll
        for (int k = 0; k < 3; ++k)
        {
          rmw[3 * dv + k] = sp[k];
          rd[3 * tv + k] = sp[k];
        }
      }
      float *mother = cps + max_id * ND * 3;
      float *dghter = cps + count * ND * 3;
      for (int t = lane; t < ND * 3; t += kWarp) dghter[t] = mother[t];
      __syncwarp ();
      // mother: split (displaced dv, tradeoff tv); daughter: the complement
      // (displaced tv, tradeoff dv); one (line, component) per lane
      for (int item = lane; item < 2 * NL * 3; item += kWarp)
      {
        const bool is_mother = item < NL * 3;
        const int it = is_mother ? item : item - NL * 3;
        const int line = it / 3;
        const int comp = it - 3 * line;
        int h = 0, g = line;
        while (g >= P - h)
        {
          g -= P - h;
          ++h;
        }
        if (is_mother) tet_split_line<P> (mother, dv, tv, g, h, comp);
        else tet_split_line<P> (dghter, tv, dv, g, h, comp);
      }
      __syncwarp ();
      warp_hull<ND> (mother, boxes + 6 * max_id, lane);
      warp_hull<ND> (dghter, boxes + 6 * count, lane);
      __syncwarp ();
    }

    const float s = (float)1.000001;
    for (int b = lane; b < NB; b += kWarp)
    {
      float bx[6];
#pragma unroll
      for (int q = 0; q < 6; ++q) bx[q] = boxes[6 * b + q];
#pragma unroll
      for (int k = 0; k < 3; ++k) scale_range (bx[2 * k], bx[2 * k + 1], s);
      const size_t o = (size_t)el * NB + b;
#pragma unroll
      for (int q = 0; q < 6; ++q) aabbs6[6 * o + q] = bx[q];
      prim_ids[o] = el;
#pragma unroll
      for (int q = 0; q < kTetRefFloats; ++q) ref_out[kTetRefFloats * o + q] = refs[kTetRefFloats * b + q];
#pragma unroll
      for (int k = 0; k < 3; ++k)
      {
        bmn[k] = fminf (bmn[k], bx[2 * k]);
        bmx[k] = fmaxf (bmx[k], bx[2 * k + 1]);
      }
    }
  }
  reduce_scene_bounds (bmn, bmx, s_bounds, warp, lane, bounds_ord);
}

// ---- simplex faces (triangles): 17 sub-boxes per triangle ----
//
// The same split with dim 2: the reference sub-triangle is three vertices
// (u and v axis vertices, then the origin), the longest of its three edges
// is halved, and split_inplace<2,Simplex> (elem_ops.hpp:1216-1250) runs de
// Casteljau along it on the rows parallel to it.  Its triangle index
// (cartesian_to_tri_idx) is the evaluators' layout, so these boxes match the
// reference's at every order.

constexpr int kTriRefFloats = 6; // SubRef<2,Simplex>: three vertices

template <int P>
DRB_D void tri_split_line (float *cps, int v0, int v1, int g, int comp)
{
  const int v2 = 3 - v0 - v1;
  const int m = P - g;
  int ids[P + 1];
  float d[P + 1];
#pragma unroll
  for (int a = 0; a <= P; ++a)
  {
    if (a > m) break;
    int b[3];
    b[v0] = a;
    b[v1] = m - a;
    b[v2] = g;
    ids[a] = tri_index (b[0], b[1], P);
    d[a] = cps[3 * ids[a] + comp];
  }
#pragma unroll
  for (int nu = P; nu >= 1; --nu)
  {
    if (nu > m) continue;
#pragma unroll
    for (int a = P; a >= 1; --a)
    {
      if (a > m || a < m - nu + 1) continue;
      d[a] = __fadd_rn (__fmul_rn (d[a], 0.5f), __fmul_rn (d[a - 1], 0.5f));
    }
  }
#pragma unroll
  for (int a = 0; a <= P; ++a)
  {
    if (a > m) break;
    cps[3 * ids[a] + comp] = d[a];
  }
}

template <int P>
__global__ void __launch_bounds__ (kSubboxWarps * kWarp)
tri_subbox_kernel (const int *__restrict__ ctrl_idx, const float *__restrict__ xyz, int n_elem,
                   float *__restrict__ aabbs6, int *__restrict__ prim_ids,
                   float *__restrict__ ref_out, unsigned *__restrict__ bounds_ord)
{
  constexpr int ND = tri_dofs<P> ();
  constexpr int NB = SplitCount<2>::boxes;
  constexpr int CPW = NB * ND * 3;
  extern __shared__ float smem[];
  __shared__ float s_bounds[kSubboxWarps][6];

  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  float *cps = smem + warp * CPW;
  float *boxes = smem + kSubboxWarps * CPW + warp * NB * 6;
  float *refs = smem + kSubboxWarps * (CPW + NB * 6) + warp * NB * kTriRefFloats;

  const int el = blockIdx.x * kSubboxWarps + warp;
  float bmn[3] = { INFINITY, INFINITY, INFINITY };
  float bmx[3] = { -INFINITY, -INFINITY, -INFINITY };

  if (el < n_elem)
  {
    for (int t = lane; t < ND * 3; t += kWarp)
    {
      const int i = t / 3;
      const int k = t - 3 * i;
      cps[t] = __ldg (xyz + 3 * (size_t)__ldg (ctrl_idx + (size_t)el * ND + i) + k);
    }
    // ref_universe<Simplex> in 2D: (1,0), (0,1), then the origin
    if (lane < kTriRefFloats) refs[lane] = (lane == 0 || lane == 3) ? 1.f : 0.f;
    __syncwarp ();
    warp_hull<ND> (cps, boxes, lane);
    __syncwarp ();

    for (int count = 1; count < NB; ++count)
    {
      int max_id = 0;
      float max_measure = box_measure (boxes);
      for (int b = 1; b < count; ++b)
      {
        const float mm = box_measure (boxes + 6 * b);
        if (mm > max_measure)
        {
          max_id = b;
          max_measure = mm;
        }
      }
      const float *rm = refs + max_id * kTriRefFloats;
      int dv = 0, tv = 1;
      float max_l2 = 0.f;
      for (int a = 0; a < 2; ++a)
        for (int b = a + 1; b < 3; ++b)
        {
          const float e0 = __fsub_rn (rm[2 * a], rm[2 * b]);
          const float e1 = __fsub_rn (rm[2 * a + 1], rm[2 * b + 1]);
          const float l2 = __fadd_rn (__fmul_rn (e0, e0), __fmul_rn (e1, e1));
          if (l2 > max_l2)
          {
            dv = a;
            tv = b;
            max_l2 = l2;
          }
        }
      __syncwarp ();
      if (lane == 0)
      {
        float *rmw = refs + max_id * kTriRefFloats;
        float *rd = refs + count * kTriRefFloats;
        float sp[2];
#pragma unroll
        for (int k = 0; k < 2; ++k)
          sp[k] = __fadd_rn (__fmul_rn (rmw[2 * tv + k], 0.5f), __fmul_rn (rmw[2 * dv + k], 0.5f));
#pragma unroll
        for (int q = 0; q < kTriRefFloats; ++q) rd[q] = rmw[q];
#pragma unroll
        for (int k = 0; k < 2; ++k)
        {
          rmw[2 * dv + k] = sp[k];
          rd[2 * tv + k] = sp[k];
        }
      }
      float *mother = cps + max_id * ND * 3;
      float *dghter = cps + count * ND * 3;
      for (int t = lane; t < ND * 3; t += kWarp) dghter[t] = mother[t];
      __syncwarp ();
      // P lines (fixed exponent g < P of the third vertex) x 3 components
      for (int item = lane; item < 2 * P * 3; item += kWarp)
      {
        const bool is_mother = item < P * 3;
        const int it = is_mother ? item : item - P * 3;
        const int g = it / 3;
        const int comp = it - 3 * g;
        if (is_mother) tri_split_line<P> (mother, dv, tv, g, comp);
        else tri_split_line<P> (dghter, tv, dv, g, comp);
      }
      __syncwarp ();
      warp_hull<ND> (mother, boxes + 6 * max_id, lane);
      warp_hull<ND> (dghter, boxes + 6 * count, lane);
      __syncwarp ();
    }

    const float s = (float)1.000001;
    for (int b = lane; b < NB; b += kWarp)
    {
      float bx[6];
#pragma unroll
      for (int q = 0; q < 6; ++q) bx[q] = boxes[6 * b + q];
#pragma unroll
      for (int k = 0; k < 3; ++k) scale_range (bx[2 * k], bx[2 * k + 1], s);
      const size_t o = (size_t)el * NB + b;
#pragma unroll
      for (int q = 0; q < 6; ++q) aabbs6[6 * o + q] = bx[q];
      prim_ids[o] = el;
#pragma unroll
      for (int q = 0; q < kTriRefFloats; ++q) ref_out[kTriRefFloats * o + q] = refs[kTriRefFloats * b + q];
#pragma unroll
      for (int k = 0; k < 3; ++k)
      {
        bmn[k] = fminf (bmn[k], bx[2 * k]);
        bmx[k] = fmaxf (bmx[k], bx[2 * k + 1]);
      }
    }
  }
  reduce_scene_bounds (bmn, bmx, s_bounds, warp, lane, bounds_ord);
}

__global__ void bounds_init_kernel (unsigned *bounds_ord)
{
  const int q = threadIdx.x;
  if (q < 6) bounds_ord[q] = (q & 1) ? float_to_ordered (-INFINITY) : float_to_ordered (INFINITY);
}

__global__ void bounds_finish_kernel (const unsigned *bounds_ord, float *bounds6)
{
  const int q = threadIdx.x;
  if (q < 6) bounds6[q] = ordered_to_float (bounds_ord[q]);
}

// get_mcodes + morton_3d (linear_bvh_builder.cpp:60-90, morton_codes.hpp:16-53)
DRB_D unsigned expand_bits32 (unsigned x)
{
  x = (x | (x << 16)) & 0x030000FFu;
  x = (x | (x << 8)) & 0x0300F00Fu;
  x = (x | (x << 4)) & 0x030C30C3u;
  x = (x | (x << 2)) & 0x09249249u;
  return x;
}

__global__ void morton_kernel (const float *__restrict__ aabbs6, int n,
                               const float *__restrict__ bounds6, unsigned *__restrict__ codes,
                               int *__restrict__ iota)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float mn[3], inv[3];
#pragma unroll
  for (int k = 0; k < 3; ++k)
  {
    mn[k] = bounds6[2 * k];
    const float ext = __fsub_rn (bounds6[2 * k + 1], bounds6[2 * k]);
    inv[k] = (ext == 0.f) ? 0.f : __fdiv_rn (1.f, ext);
  }
  unsigned e[3];
#pragma unroll
  for (int k = 0; k < 3; ++k)
  {
    const float lo = aabbs6[6 * (size_t)i + 2 * k];
    const float hi = aabbs6[6 * (size_t)i + 2 * k + 1];
    // Range::center returns NaN for an empty range (range.hpp:130-137)
    const float c = (lo > hi) ? __int_as_float (0x7fc00000) : __fmul_rn (0.5f, __fadd_rn (lo, hi));
    float x = __fmul_rn (__fsub_rn (c, mn[k]), inv[k]);
    x = fminf (fmaxf (__fmul_rn (x, 1024.0f), 0.0f), 1023.0f);
    e[k] = expand_bits32 ((unsigned)x);
  }
  codes[i] = (e[2] << 2) | (e[1] << 1) | e[0];
  if (iota) iota[i] = i;
}

// reorder (linear_bvh_builder.cpp:99-118) of AABBs and primitive ids
__global__ void gather_leaves_kernel (const int *__restrict__ perm, int n,
                                      const float *__restrict__ aabbs6,
                                      const int *__restrict__ prim_ids,
                                      float *__restrict__ leaf_aabbs6, int *__restrict__ leaf_nodes)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int src = perm[i];
#pragma unroll
  for (int q = 0; q < 6; ++q) leaf_aabbs6[6 * (size_t)i + q] = aabbs6[6 * (size_t)src + q];
  leaf_nodes[i] = prim_ids[src];
}

// delta / build_tree (linear_bvh_builder.cpp:149-251), Karras 2012.
DRB_D int karras_delta (int a, int b, int inner_size, const unsigned *__restrict__ codes)
{
  const bool out = (b < 0 || b > inner_size);
  const int bb = out ? 0 : b;
  const unsigned ac = codes[a];
  const unsigned bc = codes[bb];
  unsigned exor = ac ^ bc;
  const bool tie = (exor == 0);
  exor = tie ? ((unsigned)a ^ (unsigned)bb) : exor;
  int count = __clz (exor);
  if (tie) count += 32;
  return out ? -1 : count;
}

__global__ void karras_kernel (const unsigned *__restrict__ codes, int inner_size,
                               int *__restrict__ lchild, int *__restrict__ rchild,
                               int *__restrict__ parent)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= inner_size) return;
  const int d = (0 > (karras_delta (i, i + 1, inner_size, codes) -
                      karras_delta (i, i - 1, inner_size, codes))) ? -1 : 1;
  const int min_delta = karras_delta (i, i - d, inner_size, codes);
  int lmax = 2;
  while (karras_delta (i, i + lmax * d, inner_size, codes) > min_delta) lmax *= 2;
  int l = 0;
  for (int t = lmax / 2; t >= 1; t /= 2)
    if (karras_delta (i, i + (l + t) * d, inner_size, codes) > min_delta) l += t;
  const int j = i + l * d;
  const int delta_node = karras_delta (i, j, inner_size, codes);
  int s = 0;
  float div_factor = 2.f;
  for (int t = (int)ceilf (__fdiv_rn ((float)l, div_factor));;
       div_factor *= 2.f, t = (int)ceilf (__fdiv_rn ((float)l, div_factor)))
  {
    if (karras_delta (i, i + (s + t) * d, inner_size, codes) > delta_node) s += t;
    if (t == 1) break;
  }
  const int split = i + s * d + min (d, 0);
  if (min (i, j) == split)
  {
    parent[split + inner_size] = i;
    lchild[i] = split + inner_size;
  }
  else
  {
    parent[split] = i;
    lchild[i] = split;
  }
  if (max (i, j) == split + 1)
  {
    parent[split + inner_size + 1] = i;
    rchild[i] = split + inner_size + 1;
  }
  else
  {
    parent[split + 1] = i;
    rchild[i] = split + 1;
  }
  if (i == 0) parent[0] = -1;
}

// propagate_aabbs (linear_bvh_builder.cpp:253-317): the second thread to
// reach a node unions its children.  The fence orders a child's box store
// before the counter increment that releases the parent.
__global__ void refit_kernel (const int *__restrict__ lchild, const int *__restrict__ rchild,
                              const int *__restrict__ parent, const float *__restrict__ leaf6,
                              float *inner6, int *counters, int inner_size, int leaf_size)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= leaf_size) return;
  int node = parent[inner_size + i];
  while (node != -1)
  {
    __threadfence ();
    const int old = atomicAdd (counters + node, 1);
    if (old == 0) return;
    __threadfence ();
    const int lc = lchild[node];
    const int rc = rchild[node];
    float box[6];
    const float *lb = (lc >= inner_size) ? leaf6 + 6 * (size_t)(lc - inner_size) : inner6 + 6 * (size_t)lc;
    const float *rb = (rc >= inner_size) ? leaf6 + 6 * (size_t)(rc - inner_size) : inner6 + 6 * (size_t)rc;
#pragma unroll
    for (int k = 0; k < 3; ++k)
    {
      const float l0 = __ldcg (lb + 2 * k), l1 = __ldcg (lb + 2 * k + 1);
      const float r0 = __ldcg (rb + 2 * k), r1 = __ldcg (rb + 2 * k + 1);
      box[2 * k] = fminf (l0, r0);
      box[2 * k + 1] = fmaxf (l1, r1);
    }
#pragma unroll
    for (int q = 0; q < 6; ++q) __stcg (inner6 + 6 * (size_t)node + q, box[q]);
    node = parent[node];
  }
}

// emit (linear_bvh_builder.cpp:319-397)
__global__ void emit_kernel (const int *__restrict__ lchild, const int *__restrict__ rchild,
                             const float *__restrict__ leaf6, const float *__restrict__ inner6,
                             float4 *__restrict__ nodes, int inner_size)
{
  const int node = blockIdx.x * blockDim.x + threadIdx.x;
  if (node >= inner_size) return;
  int lc = lchild[node];
  int rc = rchild[node];
  const float *lb, *rb;
  if (lc >= inner_size)
  {
    lb = leaf6 + 6 * (size_t)(lc - inner_size);
    lc = -(lc - inner_size + 1);
  }
  else
  {
    lb = inner6 + 6 * (size_t)lc;
    lc *= 4;
  }
  if (rc >= inner_size)
  {
    rb = leaf6 + 6 * (size_t)(rc - inner_size);
    rc = -(rc - inner_size + 1);
  }
  else
  {
    rb = inner6 + 6 * (size_t)rc;
    rc *= 4;
  }
  float4 v1 = make_float4 (lb[0], lb[2], lb[4], lb[1]);
  float4 v2 = make_float4 (lb[3], lb[5], rb[0], rb[2]);
  float4 v3 = make_float4 (rb[4], rb[1], rb[3], rb[5]);
  float4 v4 = make_float4 (__int_as_float (lc), __int_as_float (rc), 0.f, 0.f);
  float4 *o = nodes + 4 * (size_t)node;
  o[0] = v1;
  o[1] = v2;
  o[2] = v3;
  o[3] = v4;
}

template <int NC>
__global__ void pack_kernel (const int *__restrict__ ctrl_idx, const float *__restrict__ vals,
                             int n_elem, int nd, int stride, float *__restrict__ packed)
{
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long total = (long long)n_elem * stride;
  if (t >= total) return;
  const int e = (int)(t / stride);
  const int r = (int)(t - (long long)e * stride);
  float v = 0.f;
  if (r < nd * NC)
  {
    const int i = r / NC;
    const int k = r - NC * i;
    v = __ldg (vals + (size_t)NC * __ldg (ctrl_idx + (size_t)e * nd + i) + k);
    // geometry rows: relative to the first control point (packed_stride)
    if (NC == 3) v = __fsub_rn (v, __ldg (vals + (size_t)NC * __ldg (ctrl_idx + (size_t)e * nd) + k));
  }
  else if (NC == 3 && r < nd * NC + 3)
  {
    v = __ldg (vals + (size_t)NC * __ldg (ctrl_idx + (size_t)e * nd) + (r - nd * NC));
  }
  packed[t] = v;
}

template <int DIM, int P> size_t subbox_smem ()
{
  constexpr int ND = (DIM == 3) ? (P + 1) * (P + 1) * (P + 1) : (P + 1) * (P + 1);
  constexpr int NB = SplitCount<DIM>::boxes;
  return sizeof (float) * kSubboxWarps * (NB * ND * 3 + NB * 6 + NB * 2 * DIM);
}

template <int P> size_t tet_subbox_smem ()
{
  constexpr int NB = SplitCount<3>::boxes;
  return sizeof (float) * kSubboxWarps * (NB * tet_dofs<P> () * 3 + NB * 6 + NB * kTetRefFloats);
}

template <int P>
int launch_tri_subbox (const drb_mesh *m, float *aabbs6, int *prim_ids, float *ref_boxes,
                       unsigned *bounds_ord, cudaStream_t s)
{
  constexpr int NB = SplitCount<2>::boxes;
  const size_t smem = sizeof (float) * kSubboxWarps * (NB * tri_dofs<P> () * 3 + NB * 6 + NB * kTriRefFloats);
  cudaFuncSetAttribute (tri_subbox_kernel<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  const int blocks = div_up (m->n_elem, kSubboxWarps);
  if (blocks > 0)
    tri_subbox_kernel<P><<<blocks, kSubboxWarps * kWarp, smem, s>>> (
    m->ctrl_idx, m->values, m->n_elem, aabbs6, prim_ids, ref_boxes, bounds_ord);
  return check_launch ("tri_subbox_kernel");
}

template <int P>
int launch_tet_subbox (const drb_mesh *m, float *aabbs6, int *prim_ids, float *ref_boxes,
                       unsigned *bounds_ord, cudaStream_t s)
{
  const size_t smem = tet_subbox_smem<P> ();
  cudaFuncSetAttribute (tet_subbox_kernel<P>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                        (int)smem);
  const int blocks = div_up (m->n_elem, kSubboxWarps);
  if (blocks > 0)
    tet_subbox_kernel<P><<<blocks, kSubboxWarps * kWarp, smem, s>>> (
    m->ctrl_idx, m->values, m->n_elem, aabbs6, prim_ids, ref_boxes, bounds_ord);
  return check_launch ("tet_subbox_kernel");
}

template <int DIM, int P>
int launch_subbox (const drb_mesh *m, float *aabbs6, int *prim_ids, float *ref_boxes,
                   unsigned *bounds_ord, cudaStream_t s)
{
  const size_t smem = subbox_smem<DIM, P> ();
  cudaFuncSetAttribute (subbox_kernel<DIM, P>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                        (int)smem);
  const int blocks = div_up (m->n_elem, kSubboxWarps);
  if (blocks > 0)
    subbox_kernel<DIM, P><<<blocks, kSubboxWarps * kWarp, smem, s>>> (
    m->ctrl_idx, m->values, m->n_elem, aabbs6, prim_ids, ref_boxes, bounds_ord);
  return check_launch ("subbox_kernel");
}

int dispatch_subbox (const drb_mesh *m, float *aabbs6, int *prim_ids, float *ref_boxes,
                     unsigned *bounds_ord, cudaStream_t s)
{
  if (m->shape == DRB_SHAPE_SIMPLEX && m->dim == 3)
  {
    if (m->order == 1) return launch_tet_subbox<1> (m, aabbs6, prim_ids, ref_boxes, bounds_ord, s);
    if (m->order == 2) return launch_tet_subbox<2> (m, aabbs6, prim_ids, ref_boxes, bounds_ord, s);
    if (m->order == 3) return launch_tet_subbox<3> (m, aabbs6, prim_ids, ref_boxes, bounds_ord, s);
  }
  else if (m->shape == DRB_SHAPE_SIMPLEX && m->dim == 2)
  {
    if (m->order == 1) return launch_tri_subbox<1> (m, aabbs6, prim_ids, ref_boxes, bounds_ord, s);
    if (m->order == 2) return launch_tri_subbox<2> (m, aabbs6, prim_ids, ref_boxes, bounds_ord, s);
    if (m->order == 3) return launch_tri_subbox<3> (m, aabbs6, prim_ids, ref_boxes, bounds_ord, s);
  }
  else if (m->shape != DRB_SHAPE_TENSOR)
  {
    set_last_error ("subbox: unknown element shape");
    return DRB_ERR_UNSUPPORTED;
  }
  else if (m->dim == 3)
  {
    if (m->order == 1) return launch_subbox<3, 1> (m, aabbs6, prim_ids, ref_boxes, bounds_ord, s);
    if (m->order == 2) return launch_subbox<3, 2> (m, aabbs6, prim_ids, ref_boxes, bounds_ord, s);
    if (m->order == 3) return launch_subbox<3, 3> (m, aabbs6, prim_ids, ref_boxes, bounds_ord, s);
  }
  else if (m->dim == 2)
  {
    if (m->order == 1) return launch_subbox<2, 1> (m, aabbs6, prim_ids, ref_boxes, bounds_ord, s);
    if (m->order == 2) return launch_subbox<2, 2> (m, aabbs6, prim_ids, ref_boxes, bounds_ord, s);
    if (m->order == 3) return launch_subbox<2, 3> (m, aabbs6, prim_ids, ref_boxes, bounds_ord, s);
  }
  set_last_error ("subbox: dim must be 2 or 3 and order 1..3");
  return DRB_ERR_UNSUPPORTED;
}

int validate_mesh (const drb_mesh *m, int want_ncomp)
{
  if (!m) { set_last_error ("mesh is NULL"); return DRB_ERR_INVALID_ARG; }
  if (m->dim != 2 && m->dim != 3) { set_last_error ("mesh dim must be 2 or 3"); return DRB_ERR_INVALID_ARG; }
  if (m->shape != DRB_SHAPE_TENSOR && m->shape != DRB_SHAPE_SIMPLEX)
  {
    set_last_error ("mesh shape must be tensor or simplex");
    return DRB_ERR_UNSUPPORTED;
  }
  if (m->order < 1 || m->order > 3) { set_last_error ("mesh order must be 1..3"); return DRB_ERR_UNSUPPORTED; }
  if (m->ncomp != want_ncomp) { set_last_error ("mesh ncomp mismatch"); return DRB_ERR_INVALID_ARG; }
  if (m->n_elem < 0 || m->n_ctrl < 0) { set_last_error ("negative mesh size"); return DRB_ERR_INVALID_ARG; }
  if (m->n_elem > 0 && (!m->ctrl_idx || !m->values)) { set_last_error ("mesh arrays are NULL"); return DRB_ERR_INVALID_ARG; }
  const long long nb = (m->dim == 3) ? 33 : 17;
  if ((long long)m->n_elem * nb >= (1ll << 31) - 1) { set_last_error ("too many sub-boxes for int32 leaf ids"); return DRB_ERR_INVALID_ARG; }
  return DRB_OK;
}

} // namespace

int mesh_nd (int dim, int order)
{
  int nd = 1;
  for (int d = 0; d < dim; ++d) nd *= (order + 1);
  return nd;
}

int mesh_nd (const drb_mesh *m)
{
  if (m->shape == DRB_SHAPE_SIMPLEX) return m->dim == 2 ? tri_dofs (m->order) : tet_dofs (m->order);
  return mesh_nd (m->dim, m->order);
}

} // namespace drb

using namespace drb;

extern "C" int drb_packed_stride (int dim, int order, int ncomp)
{
  if ((dim != 2 && dim != 3) || order < 1 || order > 3 || ncomp < 1) return -1;
  return packed_stride (mesh_nd (dim, order), ncomp);
}

extern "C" int drb_elem_dofs (int shape, int dim, int order)
{
  if (order < 1 || order > 3) return -1;
  if (shape == DRB_SHAPE_TENSOR && (dim == 2 || dim == 3)) return mesh_nd (dim, order);
  if (shape == DRB_SHAPE_SIMPLEX && dim == 3) return tet_dofs (order);
  if (shape == DRB_SHAPE_SIMPLEX && dim == 2) return tri_dofs (order);
  return -1;
}

extern "C" int drb_packed_stride_shape (int shape, int dim, int order, int ncomp)
{
  const int nd = drb_elem_dofs (shape, dim, order);
  if (nd < 0 || ncomp < 1) return -1;
  return packed_stride (nd, ncomp);
}

extern "C" int drb_ref_box_floats (int shape, int dim)
{
  if (dim != 2 && dim != 3) return -1;
  if (shape == DRB_SHAPE_TENSOR) return 2 * dim;
  if (shape == DRB_SHAPE_SIMPLEX) return dim * (dim + 1);
  return -1;
}

extern "C" int drb_pack_elements (const drb_mesh *mesh, float *packed, void *stream)
{
  if (!mesh || (mesh->ncomp != 1 && mesh->ncomp != 3)) { set_last_error ("pack: bad mesh"); return DRB_ERR_INVALID_ARG; }
  int st = validate_mesh (mesh, mesh->ncomp);
  if (st) return st;
  if (mesh->n_elem == 0) return DRB_OK;
  if (!packed) { set_last_error ("pack: output NULL"); return DRB_ERR_INVALID_ARG; }
  const int nd = mesh_nd (mesh);
  const int stride = packed_stride (nd, mesh->ncomp);
  const long long total = (long long)mesh->n_elem * stride;
  cudaStream_t s = (cudaStream_t)stream;
  const int blocks = div_up (total, 256);
  if (mesh->ncomp == 3)
    pack_kernel<3><<<blocks, 256, 0, s>>> (mesh->ctrl_idx, mesh->values, mesh->n_elem, nd, stride, packed);
  else
    pack_kernel<1><<<blocks, 256, 0, s>>> (mesh->ctrl_idx, mesh->values, mesh->n_elem, nd, stride, packed);
  return check_launch ("pack_kernel");
}

extern "C" int drb_bvh_sizes (int dim, int n_elem, int *n_inner, int *n_leaf)
{
  if ((dim != 2 && dim != 3) || n_elem < 0 || !n_inner || !n_leaf)
  {
    set_last_error ("bvh_sizes: bad arguments");
    return DRB_ERR_INVALID_ARG;
  }
  const long long nb = (dim == 3) ? SplitCount<3>::boxes : SplitCount<2>::boxes;
  long long leaves = nb * n_elem;
  if (leaves >= (1ll << 31) - 1) { set_last_error ("bvh_sizes: too many leaves"); return DRB_ERR_INVALID_ARG; }
  // 0 primitives: the reference inserts two dummy leaves (linear_bvh_builder.cpp:411-433)
  if (leaves == 0) leaves = 2;
  *n_leaf = (int)leaves;
  *n_inner = (int)leaves - 1;
  return DRB_OK;
}

extern "C" int drb_elem_subboxes (const drb_mesh *mesh, float *aabbs6, int *prim_ids,
                                  float *ref_boxes, float *bounds6, void *stream)
{
  int st = validate_mesh (mesh, 3);
  if (st) return st;
  cudaStream_t s = (cudaStream_t)stream;
  Scratch scr (s);
  unsigned *bord = scr.alloc<unsigned> (6);
  if (!bord) return status_from (scr.err);
  bounds_init_kernel<<<1, 32, 0, s>>> (bord);
  if ((st = check_launch ("bounds_init_kernel"))) return st;
  st = dispatch_subbox (mesh, aabbs6, prim_ids, ref_boxes, bord, s);
  if (st) return st;
  bounds_finish_kernel<<<1, 32, 0, s>>> (bord, bounds6);
  return check_launch ("bounds_finish");
}

extern "C" int drb_morton_codes (const float *aabbs6, int n, const float *bounds6,
                                 unsigned *codes, void *stream)
{
  if (n < 0 || (n > 0 && (!aabbs6 || !bounds6 || !codes)))
  {
    set_last_error ("morton: bad arguments");
    return DRB_ERR_INVALID_ARG;
  }
  if (n == 0) return DRB_OK;
  morton_kernel<<<div_up (n, 256), 256, 0, (cudaStream_t)stream>>> (aabbs6, n, bounds6, codes, nullptr);
  return check_launch ("morton_kernel");
}

extern "C" int drb_lbvh_build (const drb_mesh *mesh, drb_bvh *bvh, unsigned *sorted_codes,
                               void *stream)
{
  int st = validate_mesh (mesh, 3);
  if (st) return st;
  if (!bvh || !bvh->inner_nodes || !bvh->leaf_nodes || !bvh->aabb_ids || !bvh->ref_boxes)
  {
    set_last_error ("lbvh_build: bvh arrays must be allocated (see drb_bvh_sizes)");
    return DRB_ERR_INVALID_ARG;
  }
  int n_inner, n_leaf;
  st = drb_bvh_sizes (mesh->dim, mesh->n_elem, &n_inner, &n_leaf);
  if (st) return st;
  if (bvh->n_leaf != n_leaf || bvh->n_inner != n_inner)
  {
    set_last_error ("lbvh_build: bvh sizes do not match drb_bvh_sizes");
    return DRB_ERR_INVALID_ARG;
  }
  cudaStream_t s = (cudaStream_t)stream;

  if (mesh->n_elem == 0)
  {
    // Zero-primitive special case (linear_bvh_builder.cpp:411-433): two
    // point boxes at the origin, both leaves refer to primitive 0, and the
    // bounds stay empty because the reduction is skipped.
    float node[16] = { 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0 };
    const int kids[2] = { -1, -2 };
    std::memcpy (node + 12, kids, sizeof (kids));
    const int leaf[2] = { 0, 0 };
    const int ids[2] = { 0, 1 };
    const float ref3[12] = { 0, 0, 0, 1, 1, 1, 0, 0, 0, 1, 1, 1 };
    // ref_universe<Simplex>: axis vertices, then the origin
    const float tet_ref[24] = { 1, 0, 0, 0, 1, 0, 0, 0, 1, 0, 0, 0, 1, 0, 0, 0, 1, 0, 0, 0, 1, 0, 0, 0 };
    const float tri_ref[12] = { 1, 0, 0, 1, 0, 0, 1, 0, 0, 1, 0, 0 };
    const bool simplex = mesh->shape == DRB_SHAPE_SIMPLEX;
    cudaMemcpyAsync (bvh->inner_nodes, node, sizeof (node), cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync (bvh->leaf_nodes, leaf, sizeof (leaf), cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync (bvh->aabb_ids, ids, sizeof (ids), cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync (bvh->ref_boxes, simplex ? (mesh->dim == 3 ? tet_ref : tri_ref) : ref3,
                     sizeof (float) * (simplex ? 4 * mesh->dim * (mesh->dim + 1) / 2 : 4 * mesh->dim),
                     cudaMemcpyHostToDevice, s);
    if (sorted_codes) cudaMemsetAsync (sorted_codes, 0, sizeof (unsigned) * 2, s);
    const float empty[6] = { INFINITY, -INFINITY, INFINITY, -INFINITY, INFINITY, -INFINITY };
    for (int q = 0; q < 6; ++q) bvh->bounds[q] = empty[q];
    cudaError_t e = cudaStreamSynchronize (s);
    return status_from (e);
  }

  Scratch scr (s);
  const int n = n_leaf;
  float *aabbs = scr.alloc<float> ((size_t)6 * n);
  int *prim = scr.alloc<int> (n);
  unsigned *codes = scr.alloc<unsigned> (n);
  unsigned *codes_sorted = sorted_codes ? sorted_codes : scr.alloc<unsigned> (n);
  int *iota = scr.alloc<int> (n);
  float *leaf6 = scr.alloc<float> ((size_t)6 * n);
  int *lch = scr.alloc<int> (n_inner);
  int *rch = scr.alloc<int> (n_inner);
  int *par = scr.alloc<int> ((size_t)n + n_inner);
  float *inner6 = scr.alloc<float> ((size_t)6 * n_inner);
  int *counters = scr.alloc<int> (n_inner);
  unsigned *bord = scr.alloc<unsigned> (8);
  float *bounds6 = scr.alloc<float> (8);
  if (scr.err != cudaSuccess) return status_from (scr.err);

  bounds_init_kernel<<<1, 32, 0, s>>> (bord);
  if ((st = check_launch ("bounds_init_kernel"))) return st;
  st = dispatch_subbox (mesh, aabbs, prim, bvh->ref_boxes, bord, s);
  if (st) return st;
  bounds_finish_kernel<<<1, 32, 0, s>>> (bord, bounds6);
  if ((st = check_launch ("bounds_finish_kernel"))) return st;
  morton_kernel<<<div_up (n, 256), 256, 0, s>>> (aabbs, n, bounds6, codes, iota);
  if ((st = check_launch ("morton_kernel"))) return st;
  st = radix_sort_pairs (codes, iota, codes_sorted, bvh->aabb_ids, n, 30, s);
  if (st) return st;
  gather_leaves_kernel<<<div_up (n, 256), 256, 0, s>>> (bvh->aabb_ids, n, aabbs, prim, leaf6, bvh->leaf_nodes);
  if ((st = check_launch ("gather_leaves_kernel"))) return st;
  karras_kernel<<<div_up (n_inner, 256), 256, 0, s>>> (codes_sorted, n_inner, lch, rch, par);
  if ((st = check_launch ("karras_kernel"))) return st;
  cudaMemsetAsync (counters, 0, sizeof (int) * (size_t)n_inner, s);
  refit_kernel<<<div_up (n, 256), 256, 0, s>>> (lch, rch, par, leaf6, inner6, counters, n_inner, n);
  if ((st = check_launch ("refit_kernel"))) return st;
  emit_kernel<<<div_up (n_inner, 256), 256, 0, s>>> (lch, rch, leaf6, inner6, (float4 *)bvh->inner_nodes, n_inner);
  if ((st = check_launch ("emit_kernel"))) return st;
  float hb[8];
  cudaError_t e = cudaMemcpyAsync (hb, bounds6, sizeof (float) * 6, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize (s);
  if (e != cudaSuccess) { set_last_error (cudaGetErrorString (e)); return status_from (e); }
  for (int q = 0; q < 6; ++q) bvh->bounds[q] = hb[q];
  return DRB_OK;
}
