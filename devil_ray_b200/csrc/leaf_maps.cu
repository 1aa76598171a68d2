// Per-leaf linear maps for the DRB_GUESS_SUBBOX_LINEAR first guess.
//
// The reference starts each candidate's Newton solve from the centre c of
// the leaf's reference sub-box (its intent, data_model/device_mesh.hpp:
// 161-162).  A leaf covers a small part of its element, where the element
// map is close to its linearisation at c, so the first guess
//   x0 = c + J(c)^-1 (p - X(c))
// lands about one quadratic Newton step closer to the solution.  The map of
// each leaf, (c, X(c), J(c)^-1), is evaluated once per BVH by this kernel
// and read by the locate kernels as four float4 per candidate.  Hexes take
// the centre of the leaf's reference box, tets the centroid of its
// sub-simplex (subref_center, data_model/subref.hpp:39-48).  No reference
// counterpart.
#include "bernstein.cuh"
#include "drb_common.cuh"
#include "drb_internal.h"
#include "newton.cuh"
#include "simplex.cuh"

namespace drb
{
namespace
{

template <int P, bool TET, class CP>
DRB_D void write_leaf_map (const CP &cp, const float (&origin)[3], const float (&c)[3],
                           float4 *__restrict__ out)
{
  float X[3], Ju[3], Jv[3], Jw[3];
  if (TET) tet_eval_d<P, 3> (cp, c[0], c[1], c[2], X, Ju, Jv, Jw);
  else hex_eval_d<P, 3> (cp, c[0], c[1], c[2], X, Ju, Jv, Jw);
  // J: rows physical x, y, z; columns d/du, d/dv, d/dw.  Inverse by
  // cofactors in double (a once-per-leaf cost).
  const double a = Ju[0], b = Jv[0], cc = Jw[0];
  const double d = Ju[1], e = Jv[1], f = Jw[1];
  const double g = Ju[2], h = Jv[2], k = Jw[2];
  const double A = e * k - f * h, B = -(d * k - f * g), C = d * h - e * g;
  const double det = a * A + b * B + cc * C;
  float inv[9] = { 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f };
  const double scale = fabs (a) + fabs (b) + fabs (cc) + fabs (d) + fabs (e) + fabs (f) +
                       fabs (g) + fabs (h) + fabs (k);
  if (isfinite (det) && fabs (det) > 1e-12 * scale * scale * scale)
  {
    const double r = 1.0 / det;
    inv[0] = (float)(A * r);
    inv[1] = (float)(-(b * k - cc * h) * r);
    inv[2] = (float)((b * f - cc * e) * r);
    inv[3] = (float)(B * r);
    inv[4] = (float)((a * k - cc * g) * r);
    inv[5] = (float)(-(a * f - cc * d) * r);
    inv[6] = (float)(C * r);
    inv[7] = (float)(-(a * h - b * g) * r);
    inv[8] = (float)((a * e - b * d) * r);
  }
  const float x0 = X[0] + origin[0], x1 = X[1] + origin[1], x2 = X[2] + origin[2];
  out[0] = make_float4 (c[0], c[1], c[2], x0);
  out[1] = make_float4 (x1, x2, inv[0], inv[1]);
  out[2] = make_float4 (inv[2], inv[3], inv[4], inv[5]);
  out[3] = make_float4 (inv[6], inv[7], inv[8], 0.f);
}

template <int P, bool TET>
__global__ void leaf_maps_kernel (const float *__restrict__ packed, int stride,
                                  const int *__restrict__ ctrl_idx, const float *__restrict__ xyz,
                                  const int *__restrict__ leaf_nodes, const int *__restrict__ aabb_ids,
                                  const float *__restrict__ ref_boxes, int n_leaf,
                                  float4 *__restrict__ maps)
{
  constexpr int ND = TET ? tet_dofs<P> () : (P + 1) * (P + 1) * (P + 1);
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n_leaf) return;
  const int el = __ldg (leaf_nodes + k);
  float c[3];
  if (TET)
  {
    // sub-simplex vertices: origin, then the u, v, w axis vertices
    const float *rb = ref_boxes + 12 * (size_t)__ldg (aabb_ids + k);
#pragma unroll
    for (int d = 0; d < 3; ++d) c[d] = (rb[d] + rb[3 + d] + rb[6 + d] + rb[9 + d]) * 0.25f;
  }
  else
  {
    const float *rb = ref_boxes + 6 * (size_t)__ldg (aabb_ids + k);
#pragma unroll
    for (int d = 0; d < 3; ++d) c[d] = (rb[d] + rb[3 + d]) * 0.5f;
  }
  if (packed)
  {
    // packed rows hold coordinates relative to the element's first control
    // point, which follows them in the row
    const float *row = packed + (size_t)el * stride;
    const float origin[3] = { row[packed_origin (ND)], row[packed_origin (ND) + 1],
                              row[packed_origin (ND) + 2] };
    write_leaf_map<P, TET> (PackedCP{ row }, origin, c, maps + 4 * (size_t)k);
  }
  else
  {
    const float origin[3] = { 0.f, 0.f, 0.f };
    write_leaf_map<P, TET> (IndirectCP{ ctrl_idx + (size_t)el * ND, xyz, 3 }, origin, c,
                       maps + 4 * (size_t)k);
  }
}

} // namespace
} // namespace drb

using namespace drb;

extern "C" int drb_bvh_leaf_maps (const drb_mesh *mesh, const drb_bvh *bvh, float *maps, void *stream)
{
  if (!mesh || !bvh || (bvh->n_leaf > 0 && (!maps || !bvh->leaf_nodes || !bvh->aabb_ids ||
                                             !bvh->ref_boxes)))
  {
    set_last_error ("bvh_leaf_maps: bad arguments");
    return DRB_ERR_INVALID_ARG;
  }
  if ((mesh->shape != DRB_SHAPE_TENSOR && mesh->shape != DRB_SHAPE_SIMPLEX) || mesh->dim != 3 ||
      mesh->ncomp != 3 || mesh->order < 1 || mesh->order > 3)
  {
    set_last_error ("bvh_leaf_maps: needs a hex or tet geometry mesh of order 1..3");
    return DRB_ERR_UNSUPPORTED;
  }
  if (reinterpret_cast<uintptr_t> (maps) % 16)
  {
    set_last_error ("bvh_leaf_maps: maps must be 16-byte aligned");
    return DRB_ERR_INVALID_ARG;
  }
  const int n = bvh->n_leaf;
  if (n == 0) return DRB_OK;
  cudaStream_t s = (cudaStream_t)stream;
  const int stride = packed_stride (mesh_nd (mesh), 3);
  const int blocks = div_up (n, 128);
  const bool tet = mesh->shape == DRB_SHAPE_SIMPLEX;
#define DRB_LM(P, T) leaf_maps_kernel<P, T><<<blocks, 128, 0, s>>> (mesh->packed, stride, mesh->ctrl_idx, mesh->values, bvh->leaf_nodes, bvh->aabb_ids, bvh->ref_boxes, n, (float4 *)maps)
  if (tet && mesh->order == 1) DRB_LM (1, true);
  else if (tet && mesh->order == 2) DRB_LM (2, true);
  else if (tet) DRB_LM (3, true);
  else if (mesh->order == 1) DRB_LM (1, false);
  else if (mesh->order == 2) DRB_LM (2, false);
  else DRB_LM (3, false);
#undef DRB_LM
  return check_launch ("leaf_maps_kernel");
}
