// Bounding planes of each tet for the batched locate's candidate filter (no
// reference counterpart).
//
// A Bernstein element lies in the convex hull of its control points, so a
// point on the far side of a plane that has every control point behind it
// is outside the element.  Per tet the four planes are those of the faces of
// the vertex tet (outward normals, unit length), each pushed out to the
// farthest control point: n_f . x <= d_f holds on the whole element.  A
// fifth record holds the element size D (the diagonal of the control points'
// box).
//
// The persistent locate kernel skips the Newton solve of a candidate with
// n_f . p - d_f > kHullMargin * tol * D for some f.  Such a solve cannot be
// accepted: acceptance needs the last Newton step below tol and a reference
// point within tol of the simplex, which puts p within a few tol times the
// element's derivative bound (at most 3 P D) of the element, far inside
// kHullMargin * tol * D.  The filter only removes solves that fail, so the
// located cells and reference points are those of the unfiltered kernel
// (tests/test_tet_gpu.py compares them bit for bit).
#include "drb_common.cuh"
#include "drb_internal.h"
#include "simplex.cuh"

namespace drb
{
namespace
{

template <int P>
__global__ void tet_hull_kernel (const int *__restrict__ ctrl_idx, const float *__restrict__ xyz,
                                 int n_elem, float4 *__restrict__ out)
{
  constexpr int ND = tet_dofs<P> ();
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n_elem) return;
  float c[ND][3];
#pragma unroll
  for (int i = 0; i < ND; ++i)
#pragma unroll
    for (int k = 0; k < 3; ++k) c[i][k] = __ldg (xyz + 3 * (size_t)__ldg (ctrl_idx + (size_t)e * ND + i) + k);
  // vertex dofs: origin, u = 1, v = 1, w = 1
  const int vid[4] = { 0, P, (P + 1) * (P + 2) / 2 - 1, ND - 1 };
  float lo[3] = { c[0][0], c[0][1], c[0][2] }, hi[3] = { c[0][0], c[0][1], c[0][2] };
#pragma unroll
  for (int i = 1; i < ND; ++i)
#pragma unroll
    for (int k = 0; k < 3; ++k)
    {
      lo[k] = fminf (lo[k], c[i][k]);
      hi[k] = fmaxf (hi[k], c[i][k]);
    }
  const float dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
  const float diam = sqrtf (dx * dx + dy * dy + dz * dz);
#pragma unroll
  for (int f = 0; f < 4; ++f)
  {
    // face opposite vertex f
    int a = -1, b = -1, cc = -1;
#pragma unroll
    for (int q = 0; q < 4; ++q)
    {
      if (q == f) continue;
      if (a < 0) a = vid[q];
      else if (b < 0) b = vid[q];
      else cc = vid[q];
    }
    const float e1[3] = { c[b][0] - c[a][0], c[b][1] - c[a][1], c[b][2] - c[a][2] };
    const float e2[3] = { c[cc][0] - c[a][0], c[cc][1] - c[a][1], c[cc][2] - c[a][2] };
    float n[3] = { e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2],
                   e1[0] * e2[1] - e1[1] * e2[0] };
    const float len = sqrtf (n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
    float4 pl = make_float4 (0.f, 0.f, 0.f, 0.f); // degenerate face: never rejects
    if (len > 0.f && isfinite (len))
    {
#pragma unroll
      for (int k = 0; k < 3; ++k) n[k] /= len;
      const int o = vid[f];
      const float side = n[0] * (c[o][0] - c[a][0]) + n[1] * (c[o][1] - c[a][1]) +
                         n[2] * (c[o][2] - c[a][2]);
      if (side > 0.f)
#pragma unroll
        for (int k = 0; k < 3; ++k) n[k] = -n[k];
      float d = -INFINITY;
#pragma unroll
      for (int i = 0; i < ND; ++i) d = fmaxf (d, n[0] * c[i][0] + n[1] * c[i][1] + n[2] * c[i][2]);
      pl = make_float4 (n[0], n[1], n[2], d);
    }
    out[5 * (size_t)e + f] = pl;
  }
  out[5 * (size_t)e + 4] = make_float4 (diam, 0.f, 0.f, 0.f);
}

} // namespace
} // namespace drb

using namespace drb;

extern "C" int drb_tet_hull_planes (const drb_mesh *mesh, float *planes, void *stream)
{
  if (!mesh || mesh->shape != DRB_SHAPE_SIMPLEX || mesh->dim != 3 || mesh->ncomp != 3 ||
      mesh->order < 1 || mesh->order > 3 || mesh->n_elem < 0 ||
      (mesh->n_elem > 0 && (!mesh->ctrl_idx || !mesh->values || !planes)))
  {
    set_last_error ("tet_hull_planes: needs a tet geometry mesh of order 1..3 and an output array");
    return DRB_ERR_INVALID_ARG;
  }
  if (mesh->n_elem == 0) return DRB_OK;
  cudaStream_t s = (cudaStream_t)stream;
  const int b = div_up (mesh->n_elem, 128);
  float4 *o = (float4 *)planes;
  if (mesh->order == 1) tet_hull_kernel<1><<<b, 128, 0, s>>> (mesh->ctrl_idx, mesh->values, mesh->n_elem, o);
  else if (mesh->order == 2) tet_hull_kernel<2><<<b, 128, 0, s>>> (mesh->ctrl_idx, mesh->values, mesh->n_elem, o);
  else tet_hull_kernel<3><<<b, 128, 0, s>>> (mesh->ctrl_idx, mesh->values, mesh->n_elem, o);
  return check_launch ("tet_hull_kernel");
}
