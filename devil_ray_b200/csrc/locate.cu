// Point location over the LBVH: Mesh::locate / DeviceMesh::locate
// (data_model/unstructured_mesh.cpp:124-148, device_mesh.hpp:248-354).
//
// locate_kernel: one thread per point, the reference's traversal order
// (stack of 64, point-in-box test on both children, left child first, first
// converged+inside leaf wins), Newton per candidate leaf.  Orders 1-2 keep the
// candidate element's control points in registers for all Newton steps
// (one float4-vectorised read of the packed row per candidate); order 3 reads
// the packed row through L1 on every step.
#include "drb_common.cuh"
#include "drb_internal.h"
#include "newton.cuh"

namespace drb
{

// Point-in-box tests of both children of an inner node (device_mesh.hpp:262-318).
DRB_D void node_point_test (const float4 *__restrict__ nodes, int node, const float (&p)[3],
                            bool &in_left, bool &in_right)
{
  const float4 a = __ldg (nodes + node + 0);
  const float4 b = __ldg (nodes + node + 1);
  const float4 c = __ldg (nodes + node + 2);
  in_left = !(p[0] < a.x || p[1] < a.y || p[2] < a.z || p[0] > a.w || p[1] > b.x || p[2] > b.y);
  in_right = !(p[0] < b.z || p[1] < b.w || p[2] < c.x || p[0] > c.y || p[1] > c.z || p[2] > c.w);
}

struct LocateParams
{
  const float4 *nodes;
  const int *leaf_nodes;
  const int *aabb_ids;
  const float *ref_boxes;
  const float *packed;
  const int *ctrl_idx;
  const float *xyz;
  int stride;
  float tol;
  int max_steps;
  int guess_mode;
  const float *guess;
};

// Newton solve of one point in one element, choosing register-resident or
// L1-read control points by order.
template <int P>
DRB_D bool solve_in_element (const LocateParams &lp, int el, const float (&pt)[3], float (&x)[3],
                             int &steps)
{
  constexpr int ND = (P + 1) * (P + 1) * (P + 1);
  if (lp.packed)
  {
    const float *row = lp.packed + (size_t)el * lp.stride;
    if (P <= 2)
    {
      RegCP<3 * ND> r;
      load_reg_cp<P> (r, row);
      return hex_newton<P> (r, pt, x, lp.tol, lp.max_steps, steps);
    }
    PackedCP cp{ row };
    return hex_newton<P> (cp, pt, x, lp.tol, lp.max_steps, steps);
  }
  IndirectCP cp{ lp.ctrl_idx + (size_t)el * ND, lp.xyz, 3 };
  return hex_newton<P> (cp, pt, x, lp.tol, lp.max_steps, steps);
}

template <int P>
DRB_D int locate_point (const LocateParams &lp, int qi, const float (&pt)[3], float (&out_ref)[3],
                        int &iters, int &cands)
{
  int todo[kStackDepth];
  int current = 0;
  int sp = 0;
  todo[sp] = kBarrier;
  bool first_candidate = true;
  while (current != kBarrier)
  {
    if (current > -1)
    {
      bool in_l, in_r;
      node_point_test (lp.nodes, current, pt, in_l, in_r);
      if (!in_l && !in_r)
      {
        current = todo[sp];
        --sp;
      }
      else
      {
        const float4 ch = __ldg (lp.nodes + current + 3);
        const int l = __float_as_int (ch.x);
        const int r = __float_as_int (ch.y);
        current = in_l ? l : r;
        if (in_l && in_r)
        {
          // depth is bounded by the tree height; 64 covers 2^63 leaves of a
          // balanced tree and the reference uses the same fixed stack
          if (sp < kStackDepth - 1) todo[++sp] = r;
        }
      }
    }
    else
    {
      const int leaf = -current - 1;
      const int el = __ldg (lp.leaf_nodes + leaf);
      ++cands;
      float x[3];
      bool given = false;
      if (lp.guess_mode == DRB_GUESS_ZERO)
      {
        x[0] = x[1] = x[2] = 0.f;
      }
      else if (lp.guess_mode == DRB_GUESS_SUBREF_CENTER)
      {
        const float *rb = lp.ref_boxes + 6 * (size_t)__ldg (lp.aabb_ids + leaf);
#pragma unroll
        for (int d = 0; d < 3; ++d) x[d] = (rb[d] + rb[3 + d]) * 0.5f;
      }
      else if (lp.guess_mode == DRB_GUESS_GIVEN && first_candidate)
      {
#pragma unroll
        for (int d = 0; d < 3; ++d) x[d] = lp.guess[3 * (size_t)qi + d];
        given = true;
      }
      else
      {
        x[0] = x[1] = x[2] = 0.5f;
      }
      first_candidate = false;
      int steps = 0;
      bool found = solve_in_element<P> (lp, el, pt, x, steps);
      iters += steps;
      if (!found && given)
      {
        // plain Newton from the element centre is the fallback of the guess
        x[0] = x[1] = x[2] = 0.5f;
        found = solve_in_element<P> (lp, el, pt, x, steps);
        iters += steps;
      }
      if (found)
      {
        out_ref[0] = x[0];
        out_ref[1] = x[1];
        out_ref[2] = x[2];
        return el;
      }
      current = todo[sp];
      --sp;
    }
  }
  return -1;
}

template <int P>
__global__ void __launch_bounds__ (128)
locate_kernel (LocateParams lp, const float *__restrict__ pts, int n, int *__restrict__ cell,
               float *__restrict__ ref, int *__restrict__ iters_out, int *__restrict__ cands_out)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float pt[3] = { pts[3 * (size_t)i], pts[3 * (size_t)i + 1], pts[3 * (size_t)i + 2] };
  float r[3] = { -1.f, -1.f, -1.f };
  int iters = 0, cands = 0;
  const int c = locate_point<P> (lp, i, pt, r, iters, cands);
  cell[i] = c;
  if (c < 0) r[0] = r[1] = r[2] = -1.f;
  ref[3 * (size_t)i] = r[0];
  ref[3 * (size_t)i + 1] = r[1];
  ref[3 * (size_t)i + 2] = r[2];
  if (iters_out) iters_out[i] = iters;
  if (cands_out) cands_out[i] = cands;
}

} // namespace drb

using namespace drb;

extern "C" int drb_locate (const drb_mesh *mesh, const drb_bvh *bvh, const float *pts, int n,
                           const drb_newton_opts *opts, int *cell, float *ref,
                           drb_query_stats stats, void *stream)
{
  if (!mesh || !bvh || !opts || n < 0 || (n > 0 && (!pts || !cell || !ref)))
  {
    set_last_error ("locate: bad arguments");
    return DRB_ERR_INVALID_ARG;
  }
  if (mesh->dim != 3 || mesh->ncomp != 3 || mesh->order < 1 || mesh->order > 3)
  {
    set_last_error ("locate: needs a hex geometry mesh of order 1..3");
    return DRB_ERR_UNSUPPORTED;
  }
  if (opts->guess_mode == DRB_GUESS_GIVEN && !opts->guess)
  {
    set_last_error ("locate: DRB_GUESS_GIVEN needs a guess array");
    return DRB_ERR_INVALID_ARG;
  }
  if (opts->max_steps < 0 || !(opts->tol > 0.f))
  {
    set_last_error ("locate: tol must be > 0 and max_steps >= 0");
    return DRB_ERR_INVALID_ARG;
  }
  if (n == 0) return DRB_OK;
  LocateParams lp;
  lp.nodes = (const float4 *)bvh->inner_nodes;
  lp.leaf_nodes = bvh->leaf_nodes;
  lp.aabb_ids = bvh->aabb_ids;
  lp.ref_boxes = bvh->ref_boxes;
  lp.packed = mesh->packed;
  lp.ctrl_idx = mesh->ctrl_idx;
  lp.xyz = mesh->values;
  lp.stride = packed_stride ((mesh->order + 1) * (mesh->order + 1) * (mesh->order + 1), 3);
  lp.tol = opts->tol;
  lp.max_steps = opts->max_steps;
  lp.guess_mode = opts->guess_mode;
  lp.guess = opts->guess;
  cudaStream_t s = (cudaStream_t)stream;
  const int blocks = div_up (n, 128);
  if (mesh->order == 1)
    locate_kernel<1><<<blocks, 128, 0, s>>> (lp, pts, n, cell, ref, stats.iters, stats.candidates);
  else if (mesh->order == 2)
    locate_kernel<2><<<blocks, 128, 0, s>>> (lp, pts, n, cell, ref, stats.iters, stats.candidates);
  else
    locate_kernel<3><<<blocks, 128, 0, s>>> (lp, pts, n, cell, ref, stats.iters, stats.candidates);
  return check_launch ("locate_kernel");
}
