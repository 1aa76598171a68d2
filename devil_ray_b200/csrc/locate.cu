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
#include "locate.cuh"
#include "newton.cuh"

namespace drb
{

template <int P, int S>
__global__ void __launch_bounds__ (128)
locate_kernel (LocateParams lp, const float *__restrict__ pts, int n, int *__restrict__ cell,
               float *__restrict__ ref, int *__restrict__ iters_out, int *__restrict__ cands_out,
               int *__restrict__ nodes_out)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float pt[3] = { pts[3 * (size_t)i], pts[3 * (size_t)i + 1], pts[3 * (size_t)i + 2] };
  float r[3] = { -1.f, -1.f, -1.f };
  int iters = 0, cands = 0, nodes = 0;
  const int c = locate_point<P, false, S> (lp, i, pt, r, iters, cands, nodes);
  cell[i] = c;
  if (c < 0) r[0] = r[1] = r[2] = -1.f;
  ref[3 * (size_t)i] = r[0];
  ref[3 * (size_t)i + 1] = r[1];
  ref[3 * (size_t)i + 2] = r[2];
  if (iters_out) iters_out[i] = iters;
  if (cands_out) cands_out[i] = cands;
  if (nodes_out) nodes_out[i] = nodes;
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
  if (mesh->ncomp != 3 || mesh->order < 1 || mesh->order > 3 ||
      !((mesh->dim == 3 || mesh->dim == 2) &&
        (mesh->shape == DRB_SHAPE_TENSOR || mesh->shape == DRB_SHAPE_SIMPLEX)))
  {
    set_last_error ("locate: needs a hex, tet, quad or triangle geometry mesh of order 1..3");
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
  lp.wide = nullptr; // the reference's binary traversal
  lp.leaf_nodes = bvh->leaf_nodes;
  lp.aabb_ids = bvh->aabb_ids;
  lp.ref_boxes = bvh->ref_boxes;
  lp.packed = mesh->packed;
  lp.ctrl_idx = mesh->ctrl_idx;
  lp.xyz = mesh->values;
  lp.stride = packed_stride (mesh_nd (mesh), 3);
  lp.tol = opts->tol;
  lp.max_steps = opts->max_steps;
  lp.guess_mode = opts->guess_mode;
  lp.guess = opts->guess;
  lp.leaf_maps = mesh->dim == 3 ? (const float4 *)bvh->leaf_maps : nullptr;
  cudaStream_t s = (cudaStream_t)stream;
  const int blocks = div_up (n, 128);
#define DRB_LK(P, S) locate_kernel<P, S><<<blocks, 128, 0, s>>> (lp, pts, n, cell, ref, stats.iters, stats.candidates, stats.nodes)
  if (mesh->shape == DRB_SHAPE_SIMPLEX && mesh->dim == 2)
  {
    if (mesh->order == 1) DRB_LK (1, kTri2D);
    else if (mesh->order == 2) DRB_LK (2, kTri2D);
    else DRB_LK (3, kTri2D);
  }
  else if (mesh->shape == DRB_SHAPE_SIMPLEX)
  {
    if (mesh->order == 1) DRB_LK (1, kSimplex);
    else if (mesh->order == 2) DRB_LK (2, kSimplex);
    else DRB_LK (3, kSimplex);
  }
  else if (mesh->dim == 2)
  {
    if (mesh->order == 1) DRB_LK (1, kQuad2D);
    else if (mesh->order == 2) DRB_LK (2, kQuad2D);
    else DRB_LK (3, kQuad2D);
  }
  else if (mesh->order == 1) DRB_LK (1, kTensor);
  else if (mesh->order == 2) DRB_LK (2, kTensor);
  else DRB_LK (3, kTensor);
#undef DRB_LK
  return check_launch ("locate_kernel");
}
