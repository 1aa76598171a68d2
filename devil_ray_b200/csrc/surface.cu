// Boundary extraction and surface rendering of Bernstein quad faces.
//
//   MeshBoundary       extract_faces / sort_faces / unique_faces / reconstruct /
//                      extract_face_dofs (data_model/mesh_utils.cpp:98-398,
//                      filters/mesh_boundary.cpp:22-100).  The reference sorts
//                      the (sorted) face corner tuples with a host std::sort;
//                      here four stable radix passes on the tuple components
//                      (least significant first) order them lexicographically
//                      on the device.  Boundary faces have unique corner
//                      tuples, so their order -- and the output -- is identical.
//   intersect kernel   intersect_faces (rendering/surface.cpp:304-437): ordered
//                      slab traversal (closer child first), per-leaf ray-face
//                      Newton in (u, v, t) from the sub-box centre and t = near
//                      (face_intersection.hpp:96-173), closest hit wins.
//   fragments / shade  get_fragments (traceable.cpp:49-147, dim 2: field value
//                      and normalised cross of the Jacobian columns) and
//                      Traceable::shade (traceable.cpp:242-338).
#include "bernstein.cuh"
#include "drb_common.cuh"
#include "drb_internal.h"
#include "newton.cuh"
#include "simplex.cuh"

namespace drb
{
namespace
{

// ------------------------------------------------------------ boundary --

DRB_D void sort4 (int (&f)[4])
{
  // sorting network; the result equals the reference's sort4
#define DRB_SWAP(a, b) if (f[a] > f[b]) { const int t = f[a]; f[a] = f[b]; f[b] = t; }
  DRB_SWAP (0, 1) DRB_SWAP (2, 3) DRB_SWAP (0, 2) DRB_SWAP (1, 3) DRB_SWAP (1, 2)
#undef DRB_SWAP
}

// extract_faces (Hex -> Tensor), mesh_utils.cpp:192-280: six sorted corner
// tuples per element, face ids 0..5 = x, y, z, X, Y, Z.
__global__ void extract_faces_kernel (const int *__restrict__ ctrl_idx, int n_elem, int p,
                                      int4 *__restrict__ faces)
{
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n_elem) return;
  const int sy = p + 1, sz = sy * sy;
  const int *el = ctrl_idx + (size_t)sz * sy * e;
  const int c[8] = { el[0], el[p], el[sy * p], el[sy * p + p], el[sz * p], el[sz * p + p],
                     el[sz * p + sy * p], el[sz * p + sy * p + p] };
  const int idx[6][4] = { { 0, 2, 4, 6 }, { 0, 1, 4, 5 }, { 0, 1, 2, 3 },
                          { 1, 3, 5, 7 }, { 2, 3, 6, 7 }, { 4, 5, 6, 7 } };
#pragma unroll
  for (int f = 0; f < 6; ++f)
  {
    int t[4] = { c[idx[f][0]], c[idx[f][1]], c[idx[f][2]], c[idx[f][3]] };
    sort4 (t);
    faces[(size_t)6 * e + f] = make_int4 (t[0], t[1], t[2], t[3]);
  }
}

// extract_faces (Tet -> Simplex), mesh_utils.cpp:282-344: four sorted corner
// triples per tet (fourth component -1), face f opposite corner f of
// (u = 1, v = 1, w = 1, origin).
__global__ void extract_tet_faces_kernel (const int *__restrict__ ctrl_idx, int n_elem, int p,
                                          int4 *__restrict__ faces)
{
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n_elem) return;
  const int nd = tet_dofs (p);
  const int *el = ctrl_idx + (size_t)nd * e;
  const int c[4] = { el[tet_index (p, 0, 0, p)], el[tet_index (0, p, 0, p)],
                     el[tet_index (0, 0, p, p)], el[0] };
  const int idx[4][3] = { { 1, 2, 3 }, { 0, 2, 3 }, { 0, 1, 3 }, { 0, 1, 2 } };
#pragma unroll
  for (int f = 0; f < 4; ++f)
  {
    int t[3] = { c[idx[f][0]], c[idx[f][1]], c[idx[f][2]] };
#define DRB_SWAP(a, b) if (t[a] > t[b]) { const int q = t[a]; t[a] = t[b]; t[b] = q; }
    DRB_SWAP (0, 1) DRB_SWAP (1, 2) DRB_SWAP (0, 1)
#undef DRB_SWAP
    faces[(size_t)4 * e + f] = make_int4 (t[0], t[1], t[2], -1);
  }
}

__global__ void face_key_kernel (const int4 *__restrict__ faces, const int *__restrict__ perm,
                                 int n, int comp, unsigned *__restrict__ keys)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int4 f = faces[perm[i]];
  const int v = comp == 0 ? f.x : (comp == 1 ? f.y : (comp == 2 ? f.z : f.w));
  keys[i] = (unsigned)v;
}

__global__ void iota_kernel (int *a, int n)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) a[i] = i;
}

DRB_D bool same4 (int4 a, int4 b) { return a.x == b.x && a.y == b.y && a.z == b.z && a.w == b.w; }

// unique_faces (mesh_utils.cpp:145-188): a face is on the boundary when
// neither sorted neighbour has the same tuple.
__global__ void unique_flags_kernel (const int4 *__restrict__ faces, const int *__restrict__ perm,
                                     int n, int *__restrict__ flags)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int4 me = faces[perm[i]];
  bool dup = false;
  if (i > 0 && same4 (me, faces[perm[i - 1]])) dup = true;
  if (i < n - 1 && same4 (me, faces[perm[i + 1]])) dup = true;
  flags[i] = dup ? 0 : 1;
}

// reconstruct + extract_face_dofs (mesh_boundary.cpp:57-98): the quad's
// (p+1)^2 dof indices into the unchanged volume value array.
__global__ void face_dofs_kernel (const int *__restrict__ perm, const int *__restrict__ flags,
                                  const int *__restrict__ offs, int n, int p,
                                  const int *__restrict__ ctrl_idx, const int *__restrict__ field_idx,
                                  int *__restrict__ out_idx, int *__restrict__ out_field_idx,
                                  int *__restrict__ elid_faceid)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || !flags[i]) return;
  const int face_idx = offs[i];
  const int flat = perm[i];
  const int el = flat / 6;
  const int faceid = flat - 6 * el;
  const int e1 = p + 1, e2 = e1 * e1, e3 = e2 * e1;
  const int strides[3] = { 1, e1, e2 };
  const int axis = (faceid == 0 || faceid == 3) ? 0 : ((faceid == 1 || faceid == 4) ? 1 : 2);
  const int start = (faceid < 3) ? 0 : (e1 - 1) * strides[axis];
  const int major = strides[axis == 2 ? 1 : 2];
  const int minor = strides[axis == 0 ? 1 : 0];
  const size_t orig = (size_t)el * e3;
  const size_t outo = (size_t)face_idx * e2;
  for (int ii = 0; ii < e1; ++ii)
    for (int jj = 0; jj < e1; ++jj)
    {
      const size_t src = orig + start + major * ii + minor * jj;
      out_idx[outo + e1 * ii + jj] = ctrl_idx[src];
      if (out_field_idx) out_field_idx[outo + e1 * ii + jj] = field_idx[src];
    }
  if (elid_faceid)
  {
    elid_faceid[2 * face_idx] = el;
    elid_faceid[2 * face_idx + 1] = faceid;
  }
}

// reconstruct + extract_face_dofs<Simplex> (mesh_boundary.cpp:102-185): the
// triangle's dofs (ii, jj), i fastest, are the tet dofs with the face's
// opposite exponent 0, the next two following the face's axes and the
// third the rest.  The reference looks the tet dofs up with
// cartesian_to_tet_idx, which for orders >= 2 is not the layout the
// evaluators use (see lbvh.cu); here they come from the layered index, so
// at order 1 the faces are the reference's and at orders 2-3 they are the
// tets' own boundary.
__global__ void tet_face_dofs_kernel (const int *__restrict__ perm, const int *__restrict__ flags,
                                      const int *__restrict__ offs, int n, int p,
                                      const int *__restrict__ ctrl_idx,
                                      const int *__restrict__ field_idx, int *__restrict__ out_idx,
                                      int *__restrict__ out_field_idx, int *__restrict__ elid_faceid)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || !flags[i]) return;
  const int face_idx = offs[i];
  const int flat = perm[i];
  const int el = flat / 4;
  const int faceid = flat - 4 * el;
  const int nd3 = tet_dofs (p), nd2 = tri_dofs (p);
  int pi[3];
  switch (faceid)
  {
  case 0: pi[0] = 1; pi[1] = 2; pi[2] = 3; break;
  case 1: pi[0] = 0; pi[1] = 2; pi[2] = 3; break;
  case 2: pi[0] = 0; pi[1] = 1; pi[2] = 3; break;
  default: pi[0] = 0; pi[1] = 1; pi[2] = 2; break;
  }
  const size_t orig = (size_t)el * nd3;
  const size_t outo = (size_t)face_idx * nd2;
  int b[4];
  b[faceid] = 0;
  for (int jj = 0; jj <= p; ++jj)
    for (int ii = 0; ii <= p - jj; ++ii)
    {
      b[pi[1]] = jj;
      b[pi[0]] = ii;
      b[pi[2]] = p - ii - jj;
      const size_t src = orig + tet_index (b[0], b[1], b[2], p);
      out_idx[outo + tri_index (ii, jj, p)] = ctrl_idx[src];
      if (out_field_idx) out_field_idx[outo + tri_index (ii, jj, p)] = field_idx[src];
    }
  if (elid_faceid)
  {
    elid_faceid[2 * face_idx] = el;
    elid_faceid[2 * face_idx + 1] = faceid;
  }
}

// -------------------------------------------------------------- surface --

struct SurfParams
{
  const float4 *nodes;
  const int *leaf_nodes;
  const int *aabb_ids;
  const float *ref_boxes;   // 4 floats per sub-box: u0 v0 u1 v1
  const float *packed;      // packed quad rows or NULL
  const int *ctrl_idx;
  const float *xyz;
  int stride;
  float tol;
  int max_steps;
};

// TRI: a triangle face (Element<2,3,Simplex,P>), evaluated by tri_eval_d and
// tested with TriRefSpace<2>::is_inside; else a quad.
template <int P, bool TRI, class CP>
DRB_D bool face_newton (const CP &cp, const Ray &ray, float (&x)[2], float &t, float tol,
                        int max_steps, int &steps)
{
  // Intersector_RayFace::intersect_local (face_intersection.hpp:96-173)
  float prev[3] = { x[0], x[1], t };
  bool converged = false;
  steps = 0;
  const float o[3] = { ray.orig.x, ray.orig.y, ray.orig.z };
  const float d[3] = { ray.dir.x, ray.dir.y, ray.dir.z };
  while (steps < max_steps && !converged)
  {
    x[0] = fminf (1.f, fmaxf (x[0], 0.f));
    x[1] = fminf (1.f, fmaxf (x[1], 0.f));
    float X[3], Ju[3], Jv[3];
    if (TRI) tri_eval_d<P, 3> (cp, x[0], x[1], X, Ju, Jv);
    else quad_eval_d<P, 3> (cp, x[0], x[1], X, Ju, Jv);
    float J[3][3], dy[3], dx[3];
#pragma unroll
    for (int r = 0; r < 3; ++r)
    {
      dy[r] = o[r] - X[r];
      J[r][0] = Ju[r];
      J[r][1] = Jv[r];
      J[r][2] = -d[r];
    }
    LU3 lu;
    lu.factor (J);
    lu.solve (dy, dx);
    x[0] += dx[0];
    x[1] += dx[1];
    t = dx[2];
    ++steps;
    const float res = norm_linf3 (x[0] - prev[0], x[1] - prev[1], t - prev[2]);
    converged = res < tol;
    prev[0] = x[0];
    prev[1] = x[1];
    prev[2] = t;
  }
  // QuadRefSpace / TriRefSpace::is_inside without eps use epsilon<Float>() = 1e-4
  const bool inside = TRI ? is_inside_tri (x[0], x[1], kEpsilon)
                          : fminf (x[0], x[1]) >= 0.f - kEpsilon && fmaxf (x[0], x[1]) <= 1.f + kEpsilon;
  return converged && inside && ray.near_t <= t && t < ray.far_t;
}

// ---- order-1 faces: Lagae & Dutre ray/bilinear-patch test ----
// The reference intersects order-1 quads in closed form ("An Efficient
// Ray-Quadrilateral Intersection Test", Lagae and Dutre 2005;
// rendering/low_order_intersectors.hpp:20-206, used by
// FaceIntersector<Quad_P1>, rendering/surface.cpp:253-300) instead of
// Newton.  Restated with every operation rounded in the reference's order
// (Vec dot: running sum from 0; cross: a1 b2 - a2 b1, ...), on the absolute
// corner coordinates, so distances and (u, v) match its float results.
struct V3
{
  float x, y, z;
};
DRB_D V3 vsub (V3 a, V3 b) { return { __fsub_rn (a.x, b.x), __fsub_rn (a.y, b.y), __fsub_rn (a.z, b.z) }; }
DRB_D V3 vcross (V3 a, V3 b)
{
  return { __fsub_rn (__fmul_rn (a.y, b.z), __fmul_rn (a.z, b.y)),
           __fsub_rn (__fmul_rn (a.z, b.x), __fmul_rn (a.x, b.z)),
           __fsub_rn (__fmul_rn (a.x, b.y), __fmul_rn (a.y, b.x)) };
}
DRB_D float vdot (V3 a, V3 b)
{
  float r = 0.f;
  r = __fadd_rn (r, __fmul_rn (a.x, b.x));
  r = __fadd_rn (r, __fmul_rn (a.y, b.y));
  r = __fadd_rn (r, __fmul_rn (a.z, b.z));
  return r;
}

// distance (INFINITY on a miss), alpha, beta, e01, e03 of the quad
// v00 v10 v11 v01
DRB_D float ld_intersect (V3 v00, V3 v10, V3 v11, V3 v01, V3 o, V3 d, float &alpha, float &beta,
                          V3 &e01, V3 &e03)
{
  const float eps = 0.00001f;
  float distance = INFINITY;
  e03 = vsub (v01, v00);
  const V3 p = vcross (d, e03);
  e01 = vsub (v10, v00);
  const float det = vdot (e01, p);
  bool hit = true;
  const float rel_eps = __fmul_rn (__fsqrt_rn (vdot (e03, e03)), eps);
  if (fabsf (det) < rel_eps) hit = false;
  const float inv_det = __fdiv_rn (1.0f, det);
  const V3 t = vsub (o, v00);
  alpha = __fmul_rn (vdot (t, p), inv_det);
  if (alpha < 0.f) hit = false;
  const V3 q = vcross (t, e01);
  beta = __fmul_rn (vdot (d, q), inv_det);
  if (beta < 0.f) hit = false;
  if (__fadd_rn (alpha, beta) > 1.0f)
  {
    const V3 e23 = vsub (v01, v11);
    const V3 e21 = vsub (v10, v11);
    const V3 pp = vcross (d, e21);
    const float detp = vdot (e23, pp);
    if (fabsf (detp) < rel_eps) hit = false;
    const float inv_detp = __fdiv_rn (1.0f, detp);
    const V3 tp = vsub (o, v11);
    const float alpha_p = __fmul_rn (vdot (tp, pp), inv_detp);
    if (alpha_p < 0.f) hit = false;
    const V3 qp = vcross (tp, e23);
    const float beta_p = __fmul_rn (vdot (d, qp), inv_detp);
    if (beta_p < 0.f) hit = false;
  }
  if (hit) distance = __fmul_rn (vdot (e03, q), inv_det);
  return distance;
}

// bilinear (u, v) of the hit from its barycentric alpha, beta (quad_ref_point)
DRB_D void ld_ref_point (V3 v00, V3 v11, float alpha, float beta, V3 e01, V3 e03, float &u, float &v)
{
  const float eps = 0.00001f;
  float a11, b11;
  const V3 e02 = vsub (v11, v00);
  const V3 n = vcross (e01, e02);
  if (fabsf (n.x) >= fabsf (n.y) && fabsf (n.x) >= fabsf (n.z))
  {
    a11 = __fdiv_rn (__fsub_rn (__fmul_rn (e02.y, e03.z), __fmul_rn (e02.z, e03.y)), n.x);
    b11 = __fdiv_rn (__fsub_rn (__fmul_rn (e01.y, e02.z), __fmul_rn (e01.z, e02.y)), n.x);
  }
  else if (fabsf (n.y) >= fabsf (n.x) && fabsf (n.y) >= fabsf (n.z))
  {
    a11 = __fdiv_rn (__fsub_rn (__fmul_rn (e02.z, e03.x), __fmul_rn (e02.x, e03.z)), n.y);
    b11 = __fdiv_rn (__fsub_rn (__fmul_rn (e01.z, e02.x), __fmul_rn (e01.x, e02.z)), n.y);
  }
  else
  {
    a11 = __fdiv_rn (__fsub_rn (__fmul_rn (e02.x, e03.y), __fmul_rn (e02.y, e03.x)), n.z);
    b11 = __fdiv_rn (__fsub_rn (__fmul_rn (e01.x, e02.y), __fmul_rn (e01.y, e02.x)), n.z);
  }
  if (fabsf (__fsub_rn (a11, 1.0f)) < eps)
  {
    u = alpha;
    if (fabsf (__fsub_rn (b11, 1.0f)) < eps) v = beta;
    else v = __fdiv_rn (beta, __fadd_rn (__fmul_rn (u, __fsub_rn (b11, 1.0f)), 1.0f));
  }
  else if (fabsf (__fsub_rn (b11, 1.0f)) < eps)
  {
    v = beta;
    u = __fdiv_rn (alpha, __fadd_rn (__fmul_rn (v, __fsub_rn (a11, 1.0f)), 1.0f));
  }
  else
  {
    const float A = __fsub_rn (1.0f, b11);
    const float B = __fsub_rn (__fsub_rn (__fmul_rn (alpha, __fsub_rn (b11, 1.0f)),
                                          __fmul_rn (beta, __fsub_rn (a11, 1.0f))), 1.0f);
    const float Cc = alpha;
    const float D = __fsub_rn (__fmul_rn (B, B), __fmul_rn (__fmul_rn (4.0f, A), Cc));
    const float Q = __fmul_rn (-0.5f, __fadd_rn (B, __fmul_rn (B < 0.f ? -1.0f : 1.0f, __fsqrt_rn (D))));
    u = __fdiv_rn (Q, A);
    if (u < 0.f || u > 1.f) u = __fdiv_rn (Cc, Q);
    v = __fdiv_rn (beta, __fadd_rn (__fmul_rn (u, __fsub_rn (b11, 1.0f)), 1.0f));
  }
}

// intersect_tri (rendering/low_order_intersectors.hpp:228-277, Moller and
// Trumbore), used by FaceIntersector<Tri_P1> (rendering/surface.cpp:205-250):
// distance (INFINITY on a miss) and (u, v) along b - a and c - a, every
// operation rounded in the reference's order.
DRB_D float mt_intersect (V3 a, V3 b, V3 c, V3 o, V3 d, float &u, float &v)
{
  const float eps2 = 0.0001f;
  float distance = INFINITY;
  const V3 e1 = vsub (b, a);
  const V3 e2 = vsub (c, a);
  const V3 p = vcross (d, e2);
  float dot = vdot (e1, p);
  if (dot != 0.f)
  {
    dot = __fdiv_rn (1.f, dot);
    const V3 t = vsub (o, a);
    u = __fmul_rn (vdot (t, p), dot);
    if (u >= (0.f - eps2) && u <= (1.f + eps2))
    {
      const V3 q = vcross (t, e1);
      v = __fmul_rn (vdot (d, q), dot);
      if (v >= (0.f - eps2) && v <= (1.f + eps2) && !(__fadd_rn (u, v) > 1.f))
        distance = __fmul_rn (vdot (e2, q), dot);
    }
  }
  return distance;
}

// packed face rows are read like packed hex rows (PackedCP, with its
// vector row loads at orders 2 and 3)
using QuadPackedCP = PackedCP;

// intersect_AABB (surface.cpp:120-163), explicitly rounded slab arithmetic
DRB_D bool node_ray_test (const float4 *__restrict__ nodes, int node, const float (&od)[3],
                          const float (&inv)[3], float closest, float min_dist, bool &hit_l,
                          bool &hit_r)
{
  const float4 a = __ldg (nodes + node + 0);
  const float4 b = __ldg (nodes + node + 1);
  const float4 c = __ldg (nodes + node + 2);
#define DRB_S(v, k) __fsub_rn (__fmul_rn ((v), inv[k]), od[k])
  const float xmin0 = DRB_S (a.x, 0), ymin0 = DRB_S (a.y, 1), zmin0 = DRB_S (a.z, 2);
  const float xmax0 = DRB_S (a.w, 0), ymax0 = DRB_S (b.x, 1), zmax0 = DRB_S (b.y, 2);
  const float xmin1 = DRB_S (b.z, 0), ymin1 = DRB_S (b.w, 1), zmin1 = DRB_S (c.x, 2);
  const float xmax1 = DRB_S (c.y, 0), ymax1 = DRB_S (c.z, 1), zmax1 = DRB_S (c.w, 2);
#undef DRB_S
  const float min0 = fmaxf (fmaxf (fmaxf (fminf (ymin0, ymax0), fminf (xmin0, xmax0)), fminf (zmin0, zmax0)), min_dist);
  const float max0 = fminf (fminf (fminf (fmaxf (ymin0, ymax0), fmaxf (xmin0, xmax0)), fmaxf (zmin0, zmax0)), closest);
  hit_l = (max0 >= min0);
  const float min1 = fmaxf (fmaxf (fmaxf (fminf (ymin1, ymax1), fminf (xmin1, xmax1)), fminf (zmin1, zmax1)), min_dist);
  const float max1 = fminf (fminf (fminf (fmaxf (ymin1, ymax1), fmaxf (xmin1, xmax1)), fmaxf (zmin1, zmax1)), closest);
  hit_r = (max1 >= min1);
  return min0 > min1;
}

template <int P, bool TRI>
__global__ void __launch_bounds__ (128)
surface_kernel (SurfParams sp, const Ray *__restrict__ rays, int n, RayHit *__restrict__ hits,
                int *__restrict__ it_out, int *__restrict__ ca_out)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const Ray ray = rays[i];
  RayHit hit;
  hit.hit_idx = -1;
  hit.dist = 0.f;
  hit.ref[0] = hit.ref[1] = hit.ref[2] = 0.f;
  float closest = ray.far_t;
  const float min_dist = ray.near_t;
  const float inv[3] = { rcp_safe (ray.dir.x), rcp_safe (ray.dir.y), rcp_safe (ray.dir.z) };
  const float od[3] = { __fmul_rn (ray.orig.x, inv[0]), __fmul_rn (ray.orig.y, inv[1]),
                        __fmul_rn (ray.orig.z, inv[2]) };
  int todo[kStackDepth];
  int sp_ = 0;
  int cur = 0;
  todo[0] = kBarrier;
  int iters = 0, cands = 0;
  constexpr int ND = TRI ? tri_dofs<P> () : (P + 1) * (P + 1);
  while (cur != kBarrier)
  {
    if (cur > -1)
    {
      bool hl, hr;
      const bool right_closer = node_ray_test (sp.nodes, cur, od, inv, closest, min_dist, hl, hr);
      if (!hl && !hr)
      {
        cur = todo[sp_];
        --sp_;
      }
      else
      {
        const float4 ch = __ldg (sp.nodes + cur + 3);
        const int l = __float_as_int (ch.x);
        const int r = __float_as_int (ch.y);
        cur = hl ? l : r;
        if (hl && hr && sp_ < kStackDepth - 1)
        {
          if (right_closer)
          {
            cur = r;
            todo[++sp_] = l;
          }
          else
          {
            todo[++sp_] = r;
          }
        }
      }
    }
    if (cur < 0 && cur != kBarrier)
    {
      const int leaf = -cur - 1;
      const int el = __ldg (sp.leaf_nodes + leaf);
      float x[2];
      if (TRI)
      {
        // subref_center<Simplex> (subref.hpp:39-48): origin, then the axis
        // vertices, times (float)(1.0 / 3)
        const float *rb = sp.ref_boxes + 6 * (size_t)__ldg (sp.aabb_ids + leaf);
#pragma unroll
        for (int d = 0; d < 2; ++d)
          x[d] = __fmul_rn (__fadd_rn (__fadd_rn (rb[4 + d], rb[d]), rb[2 + d]), (float)(1.0 / 3));
      }
      else
      {
        const float *rb = sp.ref_boxes + 4 * (size_t)__ldg (sp.aabb_ids + leaf);
        x[0] = (rb[0] + rb[2]) * 0.5f;
        x[1] = (rb[1] + rb[3]) * 0.5f;
      }
      float t = ray.near_t;
      int steps = 0;
      ++cands;
      bool inside;
      if (TRI && P == 1)
      {
        // closed form on the absolute vertices (dofs (0,0) (1,0) (0,1))
        const int *ci = sp.ctrl_idx + (size_t)el * 3;
        V3 c[3];
#pragma unroll
        for (int k = 0; k < 3; ++k)
        {
          const float *q = sp.xyz + 3 * (size_t)__ldg (ci + k);
          c[k] = { __ldg (q), __ldg (q + 1), __ldg (q + 2) };
        }
        const V3 o = { ray.orig.x, ray.orig.y, ray.orig.z }, dd = { ray.dir.x, ray.dir.y, ray.dir.z };
        float u = 0.f, v = 0.f;
        const float dist = mt_intersect (c[0], c[1], c[2], o, dd, u, v);
        inside = false;
        if (dist != INFINITY)
        {
          x[0] = u;
          x[1] = v;
          inside = dist < ray.far_t;
          t = dist;
        }
      }
      else if (P == 1)
      {
        // closed form on the absolute corners (dofs (0,0) (1,0) (0,1) (1,1))
        const int *ci = sp.ctrl_idx + (size_t)el * 4;
        V3 c[4];
#pragma unroll
        for (int k = 0; k < 4; ++k)
        {
          const float *q = sp.xyz + 3 * (size_t)__ldg (ci + k);
          c[k] = { __ldg (q), __ldg (q + 1), __ldg (q + 2) };
        }
        float alpha, beta;
        V3 e01, e03;
        const V3 o = { ray.orig.x, ray.orig.y, ray.orig.z }, dd = { ray.dir.x, ray.dir.y, ray.dir.z };
        const float dist = ld_intersect (c[0], c[1], c[3], c[2], o, dd, alpha, beta, e01, e03);
        inside = false;
        if (dist != INFINITY)
        {
          ld_ref_point (c[0], c[3], alpha, beta, e01, e03, x[0], x[1]);
          inside = dist < ray.far_t;
          t = dist;
        }
      }
      else if (sp.packed)
      {
        // packed rows are relative to the face's first control point
        const float *row = sp.packed + (size_t)el * sp.stride;
        Ray lr = ray;
        lr.orig.x = __fsub_rn (ray.orig.x, __ldg (row + packed_origin (ND)));
        lr.orig.y = __fsub_rn (ray.orig.y, __ldg (row + packed_origin (ND) + 1));
        lr.orig.z = __fsub_rn (ray.orig.z, __ldg (row + packed_origin (ND) + 2));
        QuadPackedCP cp{ row };
        inside = face_newton<P, TRI> (cp, lr, x, t, sp.tol, sp.max_steps, steps);
      }
      else
      {
        IndirectCP cp{ sp.ctrl_idx + (size_t)el * ND, sp.xyz, 3 };
        inside = face_newton<P, TRI> (cp, ray, x, t, sp.tol, sp.max_steps, steps);
      }
      iters += steps;
      if (inside && t < closest && t > min_dist)
      {
        hit.hit_idx = el;
        hit.dist = t;
        hit.ref[0] = x[0];
        hit.ref[1] = x[1];
        hit.ref[2] = 0.f;
        closest = t;
      }
      cur = todo[sp_];
      --sp_;
    }
  }
  hits[i] = hit;
  if (it_out) it_out[i] = iters;
  if (ca_out) ca_out[i] = cands;
}

// get_fragments (traceable.cpp:49-147) for dim 2 + Traceable::shade
// (traceable.cpp:242-338) fused: one thread per ray.
template <int P, bool TRI>
__global__ void shade_kernel (const Ray *__restrict__ rays, const RayHit *__restrict__ hits, int n,
                              const float *__restrict__ geo_packed, int gstride,
                              const float *__restrict__ fld_packed, int fstride,
                              const float4 *__restrict__ tf, int tf_size, float fmin, float fmax,
                              float inv_range, const PointLight *__restrict__ lights,
                              int n_lights, int use_lighting, float *__restrict__ frag_out,
                              float4 *__restrict__ fb, float *__restrict__ depth)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const RayHit h = hits[i];
  float scalar = -1.f;
  Vec3 normal = make3 (-1.f, -1.f, -1.f);
  if (h.hit_idx > -1)
  {
    QuadPackedCP gcp{ geo_packed + (size_t)h.hit_idx * gstride };
    float X[3], Ju[3], Jv[3];
    if (TRI) tri_eval_d<P, 3> (gcp, h.ref[0], h.ref[1], X, Ju, Jv);
    else quad_eval_d<P, 3> (gcp, h.ref[0], h.ref[1], X, Ju, Jv);
    struct FCP
    {
      const float *p;
      DRB_D float operator() (int q, int) const { return __ldg (p + q); }
    } fcp{ fld_packed + (size_t)h.hit_idx * fstride };
    float F[1], Fu[1], Fv[1];
    if (TRI) tri_eval_d<P, 1> (fcp, h.ref[0], h.ref[1], F, Fu, Fv);
    else quad_eval_d<P, 1> (fcp, h.ref[0], h.ref[1], F, Fu, Fv);
    scalar = F[0];
    normal = cross (make3 (Ju[0], Ju[1], Ju[2]), make3 (Jv[0], Jv[1], Jv[2]));
    const float m = sqrtf (dot (normal, normal));
    normal = make3 (normal.x / m, normal.y / m, normal.z / m);
  }
  if (frag_out)
  {
    frag_out[4 * (size_t)i] = scalar;
    frag_out[4 * (size_t)i + 1] = normal.x;
    frag_out[4 * (size_t)i + 2] = normal.y;
    frag_out[4 * (size_t)i + 3] = normal.z;
  }
  if (h.hit_idx <= -1 || !fb) return;
  const Ray ray = rays[i];
  float s = clampf (scalar, fmin, fmax);
  const float normalized = (s - fmin) * inv_range;
  int idx = (int)(normalized * float (tf_size - 1));
  idx = min (max (idx, 0), tf_size - 1);
  const float4 c = __ldg (tf + idx);
  const int pid = ray.pixel_id;
  if (!use_lighting)
  {
    fb[pid] = c;
    if (depth) depth[pid] = h.dist;
    return;
  }
  const Vec3 look = ray.dir;
  Vec3 fn = normal;
  {
    const float m = sqrtf (dot (fn, fn));
    fn = make3 (fn.x / m, fn.y / m, fn.z / m);
  }
  const Vec3 nrm = dot (look, fn) >= 0.f ? make3 (-fn.x, -fn.y, -fn.z) : fn;
  const Vec3 hit_pt = ray.orig + look * h.dist;
  const Vec3 view = make3 (-look.x, -look.y, -look.z);
  float acc[4] = { 0.f, 0.f, 0.f, 0.f };
  const float cc[3] = { c.x, c.y, c.z };
  for (int l = 0; l < n_lights; ++l)
  {
    const PointLight L = lights[l];
    Vec3 ld = make3 (L.pos[0] - hit_pt.x, L.pos[1] - hit_pt.y, L.pos[2] - hit_pt.z);
    {
      const float m = sqrtf (dot (ld, ld));
      ld = make3 (ld.x / m, ld.y / m, ld.z / m);
    }
    const float diffuse = clampf (dot (ld, nrm), 0.f, 1.f);
    float sc[4] = { L.amb[0] * c.x, L.amb[1] * c.y, L.amb[2] * c.z, c.w };
#pragma unroll
    for (int k = 0; k < 3; ++k) sc[k] += diffuse * L.diff[k] * cc[k];
    Vec3 hv = view + ld;
    {
      const float m = sqrtf (dot (hv, hv));
      hv = make3 (hv.x / m, hv.y / m, hv.z / m);
    }
    const float doth = clampf (dot (nrm, hv), 0.f, 1.f);
    const float intensity = powf (doth, L.spec_pow);
#pragma unroll
    for (int k = 0; k < 3; ++k) sc[k] += intensity * L.spec[k] * cc[k];
#pragma unroll
    for (int k = 0; k < 4; ++k) acc[k] += sc[k];
  }
#pragma unroll
  for (int k = 0; k < 3; ++k) acc[k] = clampf (acc[k], 0.f, 1.f);
  fb[pid] = make_float4 (acc[0], acc[1], acc[2], acc[3]);
  if (depth) depth[pid] = h.dist;
}

// ray_max (ray.cpp:243-259)
// ScalarRenderer::render (rendering/scalar_renderer.cpp:296-365): per hit
// ray, the depth and zone id of the hit and the fragment's scalar go to the
// ray's pixel.
__global__ void scalar_buffer_kernel (const Ray *__restrict__ rays, const RayHit *__restrict__ hits,
                                      const float4 *__restrict__ frags, int n, int zone_offset,
                                      float *__restrict__ depths, int *__restrict__ zone_ids,
                                      float *__restrict__ scalars)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const RayHit h = hits[i];
  if (h.hit_idx <= -1) return;
  const int pid = rays[i].pixel_id;
  if (depths) depths[pid] = h.dist;
  if (zone_ids) zone_ids[pid] = h.hit_idx + zone_offset;
  if (scalars && frags) scalars[pid] = frags[i].x;
}

__global__ void ray_max_kernel (Ray *rays, const RayHit *hits, int n)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && hits[i].hit_idx != -1) rays[i].far_t = hits[i].dist;
}

} // namespace
} // namespace drb

using namespace drb;

extern "C" int drb_mesh_boundary (const drb_mesh *hex, const int *field_ctrl_idx,
                                  int *face_ctrl_idx, int *face_field_idx, int *elid_faceid,
                                  int *n_faces, void *stream)
{
  if (!hex || hex->dim != 3 || hex->order < 1 || hex->order > 3 || hex->n_elem < 0 || !n_faces ||
      (hex->shape != DRB_SHAPE_TENSOR && hex->shape != DRB_SHAPE_SIMPLEX) ||
      (hex->n_elem > 0 && !hex->ctrl_idx))
  {
    set_last_error ("mesh_boundary: needs a hex or tet mesh of order 1..3");
    return DRB_ERR_INVALID_ARG;
  }
  const bool tets = hex->shape == DRB_SHAPE_SIMPLEX;
  const int faces_per = tets ? 4 : 6;
  const long long nf = (long long)faces_per * hex->n_elem;
  if (nf >= (1ll << 31))
  {
    set_last_error ("mesh_boundary: too many faces");
    return DRB_ERR_INVALID_ARG;
  }
  if (nf == 0)
  {
    *n_faces = 0;
    return DRB_OK;
  }
  cudaStream_t s = (cudaStream_t)stream;
  const int n = (int)nf;
  Scratch scr (s);
  int4 *faces = scr.alloc<int4> (n);
  int *perm_a = scr.alloc<int> (n);
  int *perm_b = scr.alloc<int> (n);
  unsigned *keys = scr.alloc<unsigned> (n);
  unsigned *keys_out = scr.alloc<unsigned> (n);
  int *flags = scr.alloc<int> (n);
  int *offs = scr.alloc<int> (n);
  int *total = scr.alloc<int> (1);
  if (scr.err != cudaSuccess) return status_from (scr.err);
  if (tets)
    extract_tet_faces_kernel<<<div_up (hex->n_elem, 128), 128, 0, s>>> (hex->ctrl_idx, hex->n_elem, hex->order, faces);
  else
    extract_faces_kernel<<<div_up (hex->n_elem, 128), 128, 0, s>>> (hex->ctrl_idx, hex->n_elem, hex->order, faces);
  int st = check_launch ("extract_faces_kernel");
  if (st) return st;
  iota_kernel<<<div_up (n, 256), 256, 0, s>>> (perm_a, n);
  if ((st = check_launch ("iota_kernel"))) return st;
  // lexicographic order of (f0,f1,f2,f3): stable passes from the last key
  for (int comp = 3; comp >= 0; --comp)
  {
    face_key_kernel<<<div_up (n, 256), 256, 0, s>>> (faces, perm_a, n, comp, keys);
    if ((st = check_launch ("face_key_kernel"))) return st;
    if ((st = radix_sort_pairs (keys, perm_a, keys_out, perm_b, n, 32, s))) return st;
    int *t = perm_a;
    perm_a = perm_b;
    perm_b = t;
  }
  unique_flags_kernel<<<div_up (n, 256), 256, 0, s>>> (faces, perm_a, n, flags);
  if ((st = check_launch ("unique_flags_kernel"))) return st;
  if ((st = exclusive_scan_i32 (flags, offs, n, total, s))) return st;
  int h = 0;
  cudaError_t e = cudaMemcpyAsync (&h, total, sizeof (int), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize (s);
  if (e != cudaSuccess) return status_from (e);
  *n_faces = h;
  if (face_ctrl_idx && tets)
  {
    tet_face_dofs_kernel<<<div_up (n, 256), 256, 0, s>>> (perm_a, flags, offs, n, hex->order,
                                                          hex->ctrl_idx, field_ctrl_idx,
                                                          face_ctrl_idx, face_field_idx, elid_faceid);
    if ((st = check_launch ("tet_face_dofs_kernel"))) return st;
  }
  else if (face_ctrl_idx)
  {
    face_dofs_kernel<<<div_up (n, 256), 256, 0, s>>> (perm_a, flags, offs, n, hex->order,
                                                      hex->ctrl_idx, field_ctrl_idx, face_ctrl_idx,
                                                      face_field_idx, elid_faceid);
    if ((st = check_launch ("face_dofs_kernel"))) return st;
  }
  return DRB_OK;
}

extern "C" int drb_surface_intersect (const drb_mesh *faces, const drb_bvh *bvh, const void *rays,
                                      int n, float tol, int max_steps, void *hits,
                                      drb_ray_stats stats, void *stream)
{
  if (!faces || !bvh || n < 0 || (n > 0 && (!rays || !hits)))
  {
    set_last_error ("surface_intersect: bad arguments");
    return DRB_ERR_INVALID_ARG;
  }
  if (faces->dim != 2 || faces->ncomp != 3 || faces->order < 1 || faces->order > 3 ||
      (faces->shape != DRB_SHAPE_TENSOR && faces->shape != DRB_SHAPE_SIMPLEX))
  {
    set_last_error ("surface_intersect: needs a quad or triangle mesh of order 1..3");
    return DRB_ERR_UNSUPPORTED;
  }
  const bool tri = faces->shape == DRB_SHAPE_SIMPLEX;
  if (n == 0) return DRB_OK;
  SurfParams sp;
  sp.nodes = (const float4 *)bvh->inner_nodes;
  sp.leaf_nodes = bvh->leaf_nodes;
  sp.aabb_ids = bvh->aabb_ids;
  sp.ref_boxes = bvh->ref_boxes;
  sp.packed = faces->packed;
  sp.ctrl_idx = faces->ctrl_idx;
  sp.xyz = faces->values;
  sp.stride = packed_stride (mesh_nd (faces), 3);
  sp.tol = tol;
  sp.max_steps = max_steps;
  cudaStream_t s = (cudaStream_t)stream;
  const int blocks = div_up (n, 128);
#define DRB_SK(P, T) surface_kernel<P, T><<<blocks, 128, 0, s>>> (sp, (const Ray *)rays, n, (RayHit *)hits, stats.iters, stats.candidates)
  if (tri)
  {
    if (faces->order == 1) DRB_SK (1, true);
    else if (faces->order == 2) DRB_SK (2, true);
    else DRB_SK (3, true);
  }
  else if (faces->order == 1) DRB_SK (1, false);
  else if (faces->order == 2) DRB_SK (2, false);
  else DRB_SK (3, false);
#undef DRB_SK
  return check_launch ("surface_kernel");
}

extern "C" int drb_surface_shade (const drb_mesh *faces, const drb_mesh *face_field,
                                  const void *rays, const void *hits, int n, const float *tf,
                                  int tf_size, const float *range2, const void *lights,
                                  int n_lights, int use_lighting, float *fragments,
                                  float *fb_rgba, float *fb_depth, void *stream)
{
  if (!faces || !face_field || n < 0 || (n > 0 && (!hits || (fb_rgba && !rays))) || !tf || tf_size < 1 ||
      !range2 || n_lights < 0 || (n_lights > 0 && !lights))
  {
    set_last_error ("surface_shade: bad arguments");
    return DRB_ERR_INVALID_ARG;
  }
  if (!faces->packed || !face_field->packed || faces->order != face_field->order ||
      faces->dim != 2 || face_field->ncomp != 1 || faces->shape != face_field->shape ||
      (faces->shape != DRB_SHAPE_TENSOR && faces->shape != DRB_SHAPE_SIMPLEX))
  {
    set_last_error ("surface_shade: needs packed quad (or triangle) geometry and scalar field "
                    "of one order");
    return DRB_ERR_INVALID_ARG;
  }
  if (n == 0) return DRB_OK;
  const int nd = mesh_nd (faces);
  const bool tri = faces->shape == DRB_SHAPE_SIMPLEX;
  const float fmin = range2[0], fmax = range2[1];
  float len = fmax - fmin;
  const float g = (fabsf (len) < 1e-8f) ? (std::signbit (len) ? -1e-8f : 1e-8f) : len;
  const float inv_range = 1.0f / g;
  cudaStream_t s = (cudaStream_t)stream;
  const int blocks = div_up (n, 128);
#define DRB_SHADE(P, T)                                                                                \
  shade_kernel<P, T><<<blocks, 128, 0, s>>> ((const Ray *)rays, (const RayHit *)hits, n, faces->packed, \
                                          packed_stride (nd, 3), face_field->packed,                 \
                                          packed_stride (nd, 1), (const float4 *)tf, tf_size, fmin,  \
                                          fmax, inv_range, (const PointLight *)lights, n_lights,     \
                                          use_lighting, fragments, (float4 *)fb_rgba, fb_depth)
  if (tri)
  {
    if (faces->order == 1) DRB_SHADE (1, true);
    else if (faces->order == 2) DRB_SHADE (2, true);
    else DRB_SHADE (3, true);
  }
  else if (faces->order == 1) DRB_SHADE (1, false);
  else if (faces->order == 2) DRB_SHADE (2, false);
  else DRB_SHADE (3, false);
#undef DRB_SHADE
  return check_launch ("shade_kernel");
}

extern "C" int drb_ray_max (void *rays, const void *hits, int n, void *stream)
{
  if (n < 0 || (n > 0 && (!rays || !hits)))
  {
    set_last_error ("ray_max: bad arguments");
    return DRB_ERR_INVALID_ARG;
  }
  if (n == 0) return DRB_OK;
  ray_max_kernel<<<div_up (n, 256), 256, 0, (cudaStream_t)stream>>> ((Ray *)rays, (const RayHit *)hits, n);
  return check_launch ("ray_max_kernel");
}

extern "C" int drb_scalar_buffer_write (const void *rays, const void *hits, const float *frags4,
                                        int n, int zone_offset, float *depths, int *zone_ids,
                                        float *scalars, void *stream)
{
  if (n < 0 || (n > 0 && (!rays || !hits)) || (scalars && !frags4))
  {
    set_last_error ("scalar_buffer_write: bad arguments");
    return DRB_ERR_INVALID_ARG;
  }
  if (n == 0) return DRB_OK;
  scalar_buffer_kernel<<<div_up (n, 256), 256, 0, (cudaStream_t)stream>>> (
  (const Ray *)rays, (const RayHit *)hits, (const float4 *)frags4, n, zone_offset, depths, zone_ids,
  scalars);
  return check_launch ("scalar_buffer_kernel");
}
