// Face neighbours of a hex or tet mesh: for every element and each of its
// faces (hex: u=0, u=1, v=0, v=1, w=0, w=1; tet: u=0, v=0, w=0, u+v+w=1),
// the element on the other side, or -1 on the boundary.  Two faces are the
// same face when their corner control points are the same (the rule
// MeshBoundary uses to find the unshared faces, mesh_utils.cpp:98-398).
// The volume march uses the table to follow a ray from element to element
// across faces instead of going back to the BVH at every element crossing.
//
//   face_key_kernel   per face: sorted corner indices; key = the smallest
//   (radix sort of the keys, 30 bits)
//   face_match_kernel faces with equal keys are compared in full; a match
//                     links the two elements
#include "drb_common.cuh"
#include "drb_internal.h"
#include "simplex.cuh"

namespace drb
{
namespace
{

// faces sharing a smallest corner: at most 12 in a hex mesh, a few dozen
// around a vertex shared by many tets; the scan stops at the end of a group
constexpr int kMaxGroupScan = 256;

__global__ void face_key_kernel (const int *__restrict__ ctrl_idx, int n_elem, int p,
                                 unsigned *__restrict__ keys, int *__restrict__ face_id,
                                 int4 *__restrict__ rest)
{
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 6ll * n_elem) return;
  const int e = (int)(t / 6), f = (int)(t - 6ll * e);
  const int axis = f >> 1, side = (f & 1) * p;
  const int n1 = p + 1, nd = n1 * n1 * n1;
  int c[4];
  int k = 0;
#pragma unroll
  for (int s = 0; s < 2; ++s)
#pragma unroll
    for (int r = 0; r < 2; ++r)
    {
      int abc[3];
      abc[axis] = side;
      abc[(axis + 1) % 3] = s * p;
      abc[(axis + 2) % 3] = r * p;
      const int dof = (abc[2] * n1 + abc[1]) * n1 + abc[0];
      c[k++] = __ldg (ctrl_idx + (size_t)e * nd + dof);
    }
  // sort the four corner indices (network of 5 compare-exchanges)
#define DRB_CX(a, b) { const int lo = min (c[a], c[b]), hi = max (c[a], c[b]); c[a] = lo; c[b] = hi; }
  DRB_CX (0, 1) DRB_CX (2, 3) DRB_CX (0, 2) DRB_CX (1, 3) DRB_CX (1, 2)
#undef DRB_CX
  keys[t] = (unsigned)c[0];
  face_id[t] = (int)t;
  rest[t] = make_int4 (c[1], c[2], c[3], 0);
}

// Tet faces: the corners are the dofs (p,0,0), (0,p,0), (0,0,p) and
// (0,0,0) of the (i, j, k) layout; face f leaves out the u, v, w vertex
// (f = 0, 1, 2) or the origin (f = 3).
__global__ void tet_face_key_kernel (const int *__restrict__ ctrl_idx, int n_elem, int p,
                                     unsigned *__restrict__ keys, int *__restrict__ face_id,
                                     int4 *__restrict__ rest)
{
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 4ll * n_elem) return;
  const int e = (int)(t / 4), f = (int)(t - 4ll * e);
  const int nd = tet_dofs (p);
  const int *row = ctrl_idx + (size_t)e * nd;
  const int U = __ldg (row + p), V = __ldg (row + tet_index (0, p, 0, p)), W = __ldg (row + nd - 1),
            O = __ldg (row);
  int c[3];
  if (f == 0) c[0] = V, c[1] = W, c[2] = O;
  else if (f == 1) c[0] = U, c[1] = W, c[2] = O;
  else if (f == 2) c[0] = U, c[1] = V, c[2] = O;
  else c[0] = U, c[1] = V, c[2] = W;
#define DRB_CX(a, b) { const int lo = min (c[a], c[b]), hi = max (c[a], c[b]); c[a] = lo; c[b] = hi; }
  DRB_CX (0, 1) DRB_CX (1, 2) DRB_CX (0, 1)
#undef DRB_CX
  keys[t] = (unsigned)c[0];
  face_id[t] = (int)t;
  rest[t] = make_int4 (c[1], c[2], 0, 0);
}

__global__ void face_match_kernel (const unsigned *__restrict__ skeys, const int *__restrict__ sface,
                                   const int4 *__restrict__ rest, long long n_faces, int fpe,
                                   int *__restrict__ neighbors)
{
  const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n_faces) return;
  const unsigned key = skeys[j];
  const int fa = sface[j];
  const int4 ra = rest[fa];
  for (int q = 1; q <= kMaxGroupScan && j + q < n_faces; ++q)
  {
    if (skeys[j + q] != key) break;
    const int fb = sface[j + q];
    const int4 rb = rest[fb];
    if (ra.x == rb.x && ra.y == rb.y && ra.z == rb.z && fa / fpe != fb / fpe)
    {
      neighbors[fa] = fb / fpe;
      neighbors[fb] = fa / fpe;
      break;
    }
  }
}

} // namespace
} // namespace drb

using namespace drb;

extern "C" int drb_mesh_face_neighbors (const drb_mesh *mesh, int *neighbors, void *stream)
{
  if (!mesh || mesh->dim != 3 || mesh->order < 1 || mesh->order > 3 || mesh->n_elem < 0 ||
      (mesh->shape != DRB_SHAPE_TENSOR && mesh->shape != DRB_SHAPE_SIMPLEX) ||
      (mesh->n_elem > 0 && (!mesh->ctrl_idx || !neighbors)))
  {
    set_last_error ("mesh_face_neighbors: needs a hex or tet mesh of order 1..3 and an output array");
    return DRB_ERR_INVALID_ARG;
  }
  const bool tet = mesh->shape == DRB_SHAPE_SIMPLEX;
  const int fpe = tet ? 4 : 6;
  if (mesh->n_elem == 0) return DRB_OK;
  if (mesh->n_ctrl > (1 << 30) || (long long)fpe * mesh->n_elem > (1ll << 31) - 1)
  {
    set_last_error ("mesh_face_neighbors: mesh too large (2^30 control points, 2^31 faces)");
    return DRB_ERR_INVALID_ARG;
  }
  cudaStream_t s = (cudaStream_t)stream;
  const int nf = fpe * mesh->n_elem;
  Scratch scr (s);
  unsigned *keys = scr.alloc<unsigned> (nf);
  unsigned *skeys = scr.alloc<unsigned> (nf);
  int *fid = scr.alloc<int> (nf);
  int *sfid = scr.alloc<int> (nf);
  int4 *rest = scr.alloc<int4> (nf);
  if (!rest) return status_from (scr.err);
  cudaMemsetAsync (neighbors, 0xFF, sizeof (int) * (size_t)nf, s); // -1: boundary
  if (tet)
    tet_face_key_kernel<<<div_up (nf, 256), 256, 0, s>>> (mesh->ctrl_idx, mesh->n_elem, mesh->order,
                                                         keys, fid, rest);
  else
    face_key_kernel<<<div_up (nf, 256), 256, 0, s>>> (mesh->ctrl_idx, mesh->n_elem, mesh->order,
                                                       keys, fid, rest);
  int st = check_launch ("face_key_kernel");
  if (st) return st;
  if ((st = radix_sort_pairs (keys, fid, skeys, sfid, nf, 30, s))) return st;
  face_match_kernel<<<div_up (nf, 256), 256, 0, s>>> (skeys, sfid, rest, nf, fpe, neighbors);
  return check_launch ("face_match_kernel");
}
